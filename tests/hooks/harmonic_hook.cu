// harmonic_hook.cu — a force consumer installed through the device force-hook
// ABI (soil_sys_set_force_hook), written the way an external physics tier
// would: it only sees the soil_dev_view.  It recomputes the tutorial's
// soft_repulsion_force over the CSR half list with atomic scatter (so its
// summation order, unlike the built-in consumer's, is not the reference's)
// and zeroes every force first.  Built by the GPU tests with nvcc; test code,
// not part of the library.
#include <cuda_runtime.h>

#include "soil_cuda.h"

namespace {

__global__ void zero_forces(soil_dev_view v) {
    const uint64_t n = v.nlocal + v.nghost;
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n;
         a += (uint64_t)gridDim.x * blockDim.x) {
        v.fx[a] = 0.0;
        v.fy[a] = 0.0;
        v.fz[a] = 0.0;
    }
}

__global__ void pair_forces(soil_dev_view v, double K) {
    const double* rad = v.columns[0];  // registered column 0: the radius
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < v.nlocal;
         i += (uint64_t)gridDim.x * blockDim.x) {
        for (uint32_t p = v.neighbor_offsets[i]; p < v.neighbor_offsets[i + 1]; ++p) {
            const uint32_t j = v.neighbor_indices[p];
            const double sum_r = rad[i] + rad[j];
            const double dx = v.x[j] - v.x[i], dy = v.y[j] - v.y[i], dz = v.z[j] - v.z[i];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 >= sum_r * sum_r || d2 == 0.0) continue;
            const double d = sqrt(d2);
            const double fm = K * (sum_r - d);
            const double fx = -fm * dx / d, fy = -fm * dy / d, fz = -fm * dz / d;
            atomicAdd(&v.fx[i], fx);
            atomicAdd(&v.fy[i], fy);
            atomicAdd(&v.fz[i], fz);
            if (v.newton || j < v.nlocal) {
                atomicAdd(&v.fx[j], -fx);
                atomicAdd(&v.fy[j], -fy);
                atomicAdd(&v.fz[j], -fz);
            }
        }
    }
}

}  // namespace

// user: pointer to the spring constant K (a double)
extern "C" int harmonic_hook(const soil_dev_view* v, void* user) {
    const double K = *static_cast<const double*>(user);
    cudaStream_t st = static_cast<cudaStream_t>(v->stream);
    zero_forces<<<592, 256, 0, st>>>(*v);
    pair_forces<<<592, 256, 0, st>>>(*v, K);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// a hook that reports failure (the step must return an error, not continue)
extern "C" int failing_hook(const soil_dev_view*, void*) { return 7; }
