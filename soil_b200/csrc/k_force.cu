// k_force.cu — the built-in pair consumer: linear repulsion
// f = k*overlap along the line of centres, the tutorial's
// soft_repulsion_force (docs/src/tutorial/write-your-own-physics.md:56-110).
//
// The reference accumulates pair forces in global pair order: for pair
// (i, j) it adds +f to i and -f to j, rows ascending, CSR order inside a row.
// So atom a receives, in order, -f(i,a) from every earlier row i that lists
// a (ascending i), then +f(a,j) for its own row, then (full lists only) -f
// from later rows.  This kernel gathers exactly that sequence per atom from
// the CSR and its transpose — one thread per atom, no atomics — so the sums
// are bit-identical to the sequential reference.  f(i,j) is always evaluated
// with i the row atom, so both endpoints recompute the same value.
#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

__global__ void __launch_bounds__(kBlock, 5) k_harmonic(uint64_t nlocal, uint64_t ntotal, AtomCols c,
                                                     const double* rad, double K, int newton,
                                                     const uint32_t* offsets,
                                                     const uint32_t* indices,
                                                     const uint32_t* in_start,
                                                     const uint32_t* in_list) {
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < ntotal;
         a += (uint64_t)gridDim.x * blockDim.x)
        harmonic_atom(c, a, nlocal, rad, K, newton, offsets, indices, in_start, in_list);
}

void launch_harmonic(cudaStream_t st, uint64_t nlocal, uint64_t ntotal, const AtomCols& c,
                     const double* radius, double k, int newton, const uint32_t* offsets,
                     const uint32_t* indices, const uint32_t* in_start, const uint32_t* in_list) {
    if (ntotal == 0) return;
    note_launch();
    // one resident wave (5 blocks of 256 per SM at <= 48 registers), grid-stride
    const unsigned full = 148u * 5u;
    const unsigned need = (unsigned)((ntotal + kBlock - 1) / kBlock);
    k_harmonic<<<need < full ? need : full, kBlock, 0, st>>>(nlocal, ntotal, c, radius, k, newton,
                                                              offsets, indices, in_start, in_list);
}

}  // namespace soil
