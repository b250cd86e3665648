// gather_hook.cu — an external consumer built on include/soil_consumer.cuh:
// one thread per atom gathers its force in the reference's order.  Built by
// the GPU tests (with -fmad=false); test code, not part of the library.
#include <cuda_runtime.h>

#include "soil_consumer.cuh"

namespace {

__global__ void gather_forces(soil_dev_view v, double K) {
    const soil_harmonic_pair pair{v.x, v.y, v.z, v.columns[0], K};
    const uint64_t n = v.nlocal + v.nghost;
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n;
         a += (uint64_t)gridDim.x * blockDim.x) {
        double F[3];
        soil_gather_force(v, a, pair, F);
        v.fx[a] = F[0];
        v.fy[a] = F[1];
        v.fz[a] = F[2];
    }
}

}  // namespace

// user: pointer to the spring constant K (a double)
extern "C" int gather_harmonic_hook(const soil_dev_view* v, void* user) {
    if (!v->in_start || !v->in_list) return 2;
    gather_forces<<<592, 256, 0, static_cast<cudaStream_t>(v->stream)>>>(
        *v, *static_cast<const double*>(user));
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
