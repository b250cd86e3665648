// k_slots.cu — persistent per-neighbor slots move with their atom when the
// spatial sort permutes the locals: each slot row (tags, then payload) is
// gathered through the sort's permutation, like every AtomData column.
#include <algorithm>

#include "kernels.cuh"

namespace soil {

template <class T>
__global__ void k_row_gather(uint64_t n_elems, uint32_t row, const uint32_t* perm, const T* src,
                             T* dst) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n_elems;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = e / row, k = e - r * row;
        dst[e] = src[(uint64_t)perm[r] * row + k];
    }
}

void launch_slot_gather(cudaStream_t st, uint64_t n, const uint32_t* perm, uint32_t max,
                        uint32_t width, const uint32_t* src_tag, const double* src_val,
                        uint32_t* dst_tag, double* dst_val) {
    if (n == 0) return;
    const uint64_t nt = n * max, nv = nt * width;
    const unsigned cap = 148u * 16u;
    note_launch();
    k_row_gather<uint32_t><<<(unsigned)std::min<uint64_t>((nt + kBlock - 1) / kBlock, cap), kBlock,
                             0, st>>>(nt, max, perm, src_tag, dst_tag);
    note_launch();
    k_row_gather<double><<<(unsigned)std::min<uint64_t>((nv + kBlock - 1) / kBlock, cap), kBlock, 0,
                           st>>>(nv, max * width, perm, src_val, dst_val);
}

}  // namespace soil
