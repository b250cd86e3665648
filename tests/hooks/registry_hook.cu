// registry_hook.cu — a consumer that writes registered columns of every flag
// class, the device counterpart of the CPU oracle's column probe.  Built by
// the GPU tests (with -fmad=false); test code, not part of the library.
//
// Per step it gathers the harmonic pair forces in the reference's order
// (soil_gather_force), then, atom by atom:
//   every atom a (locals and ghosts): rev[a] += {0.5 x, y - z};
//                                     zacc[a] += 0.25 x
//   every local a:                    fwd[a][k] += 0.001 pos[a][k]
// Column c component k of atom i is columns[c][k * stride + i].
#include <cuda_runtime.h>

#include "soil_consumer.cuh"

struct registry_probe {
    double K;
    int32_t rev, zero, fwd;  // column indices (-1: unused); radius is column 0
};

namespace {

__global__ void probe_kernel(soil_dev_view v, registry_probe p) {
    const soil_harmonic_pair pair{v.x, v.y, v.z, v.columns[0], p.K};
    const uint64_t n = v.nlocal + v.nghost;
    const uint64_t S = v.stride;
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n;
         a += (uint64_t)gridDim.x * blockDim.x) {
        double F[3];
        soil_gather_force(v, a, pair, F);
        v.fx[a] = F[0];
        v.fy[a] = F[1];
        v.fz[a] = F[2];
        const double x = v.x[a], y = v.y[a], z = v.z[a];
        if (p.rev >= 0) {
            double* r = v.columns[p.rev];
            r[a] = r[a] + 0.5 * x;
            r[S + a] = r[S + a] + (y - z);
        }
        if (p.zero >= 0) {
            double* q = v.columns[p.zero];
            q[a] = q[a] + 0.25 * x;
        }
        if (p.fwd >= 0 && a < v.nlocal) {
            double* f = v.columns[p.fwd];
            f[a] = f[a] + 0.001 * x;
            f[S + a] = f[S + a] + 0.001 * y;
            f[2 * S + a] = f[2 * S + a] + 0.001 * z;
        }
    }
}

}  // namespace

// user: pointer to a registry_probe
extern "C" int registry_hook(const soil_dev_view* v, void* user) {
    if (!v->in_start || !v->in_list) return 2;
    probe_kernel<<<592, 256, 0, static_cast<cudaStream_t>(v->stream)>>>(
        *v, *static_cast<const registry_probe*>(user));
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
