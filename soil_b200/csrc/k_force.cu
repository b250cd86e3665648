// k_force.cu — the built-in pair consumer: linear repulsion
// f = k*overlap along the line of centres, the tutorial's
// soft_repulsion_force (docs/src/tutorial/write-your-own-physics.md:56-110).
//
// The reference accumulates pair forces in global pair order: for pair
// (i, j) it adds +f to i and -f to j, rows ascending, CSR order inside a row.
// So atom a receives, in order, -f(i,a) from every earlier row i that lists
// a (ascending i), then +f(a,j) for its own row, then (full lists only) -f
// from later rows.
//
// Two kernels reproduce that sum bit for bit:
//
//  k_harmonic   one thread per atom walks the CSR and its transpose
//               (harmonic_atom); used by the batched engine and by systems
//               whose locals can have more than 7 ghost images.
//
//  k_force_seq  the single-system consumer.  At every rebuild each atom's
//               contributions are merged into one partner sequence in the
//               reference's order (k_seq_fill).  IEEE negation is exact, so
//               f(i,j) = -f(j,i) bit for bit (d -> -d flips the sign of every
//               factor that carries it; every other factor is symmetric) and
//               F - f(i,a) is F + f(a,i): each entry is evaluated as
//               f(a, partner) and added.  The sequences are grouped by local
//               root: root t's sequence, then those of its ghost images in
//               reverse-comm fold order.  A warp takes 32 consecutive roots
//               and spreads the union of their groups over its lanes in
//               chunks (every lane busy, U independent gathers in flight per
//               lane); pair forces go to shared memory, and each lane then
//               adds its own group's entries in order, writes the forces of
//               its root and images and, with FOLD, folds the images into the
//               root exactly as reverse_send_force does (fold_root), so
//               reverse comm needs no pass of its own (force_ops.cuh).
#include "device_ops.cuh"
#include "force_ops.cuh"
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

// ---- the grouped partner sequences (rebuilt with the lists) ----------------

// Entries of atom a in the reference sum: its in-list (when it receives:
// newton, or a local) and its own row (locals).
__device__ __forceinline__ uint32_t seq_len(uint64_t a, uint64_t nlocal, int newton,
                                            const uint32_t* offsets, const uint32_t* in_start) {
    const bool local = a < nlocal;
    const uint32_t nin = (newton || local) ? in_start[a + 1] - in_start[a] : 0u;
    const uint32_t nrow = local ? offsets[a + 1] - offsets[a] : 0u;
    return nin + nrow;
}

// cnt[a] = entries of atom a (every atom); grp[t] = entries of root t's group
// (t and its images), t < nlocal.
__global__ void __launch_bounds__(kBlock) k_seq_count(SeqArgs q, uint32_t* cnt, uint32_t* grp) {
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < q.ntotal;
         a += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t n = seq_len(a, q.nlocal, q.newton, q.offsets, q.in_start);
        cnt[a] = n;
        if (a < q.nlocal) {
            uint32_t g = n;
            for (uint32_t f = q.fold_start[a]; f < q.fold_start[a + 1]; ++f)
                g += seq_len(q.nlocal + q.fold_list[f], q.nlocal, q.newton, q.offsets, q.in_start);
            grp[a] = g;
        }
    }
}

// The entries of atom a from position k on: in-list rows below a
// (ascending), a's own row in CSR order, then the in-list rows above a.
__device__ __forceinline__ uint32_t seq_put(const SeqArgs& q, uint64_t a, uint32_t k,
                                            uint8_t meta, uint32_t* seq, uint8_t* owner) {
    const bool local = a < q.nlocal;
    const uint32_t qs = q.in_start[a];
    const uint32_t nin = (q.newton || local) ? q.in_start[a + 1] - qs : 0u;
    const uint32_t rs = local ? q.offsets[a] : 0u;
    const uint32_t nrow = local ? q.offsets[a + 1] - rs : 0u;
    uint32_t i = 0;
    for (; i < nin && q.in_list[qs + i] < (uint32_t)a; ++i, ++k) {
        seq[k] = q.in_list[qs + i];
        owner[k] = meta;
    }
    for (uint32_t r = 0; r < nrow; ++r, ++k) {
        seq[k] = q.indices[rs + r];
        owner[k] = meta;
    }
    for (; i < nin; ++i, ++k) {
        seq[k] = q.in_list[qs + i];
        owner[k] = meta;
    }
    return k;
}

// Group of root t at grp_start[t]: t's entries, then each image's in fold
// order.  owner[k] = (t & 31) | item << 5: item 0 = the root, item j = its
// j-th image (at most 7 images per root, which the host checks).
__global__ void __launch_bounds__(kBlock) k_seq_fill(SeqArgs q, const uint32_t* grp_start,
                                                     uint32_t* seq, uint8_t* owner) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < q.nlocal;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t lane = (uint8_t)(t & 31);
        uint32_t k = seq_put(q, t, grp_start[t], lane, seq, owner);
        const uint32_t f0 = q.fold_start[t], f1 = q.fold_start[t + 1];
        for (uint32_t f = f0; f < f1; ++f)
            k = seq_put(q, q.nlocal + q.fold_list[f], k, (uint8_t)(lane | ((f - f0 + 1) << 5)), seq,
                        owner);
    }
}

void launch_seq_count(cudaStream_t st, const SeqArgs& q, uint32_t* cnt, uint32_t* grp) {
    if (q.ntotal == 0) return;
    note_launch();
    k_seq_count<<<grid_for(q.ntotal), kBlock, 0, st>>>(q, cnt, grp);
}

void launch_seq_fill(cudaStream_t st, const SeqArgs& q, const uint32_t* grp_start, uint32_t* seq,
                     uint8_t* owner) {
    if (q.nlocal == 0) return;
    note_launch();
    k_seq_fill<<<grid_for(q.nlocal), kBlock, 0, st>>>(q, grp_start, seq, owner);
}

// ---- the warp-cooperative consumer, one launch --------------------------------

template <int U, bool FOLD>
__global__ void __launch_bounds__(kBlock, 4) k_force_seq(ForceArgs p) {
    __shared__ ForceSmem<U> sm;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint64_t ntiles = (p.nlocal + 31) / 32;
    for (uint64_t w = (uint64_t)blockIdx.x * kForceWarps + wib; w < ntiles;
         w += (uint64_t)gridDim.x * kForceWarps)
        force_tile<U, FOLD>(p, w, sm, lane, wib);
}

void launch_force_seq(cudaStream_t st, const ForceArgs& p, bool fold) {
    if (p.nlocal == 0) return;
    note_launch();
    constexpr int U = 4;
    const uint64_t ntiles = (p.nlocal + 31) / 32;
    const uint64_t need = (ntiles + kForceWarps - 1) / kForceWarps;
    const uint64_t full = 148ull * 4ull;  // one resident wave, grid-stride over the tiles
    const unsigned grid = (unsigned)(need < full ? need : full);
    if (fold) k_force_seq<U, true><<<grid, kBlock, 0, st>>>(p);
    else k_force_seq<U, false><<<grid, kBlock, 0, st>>>(p);
}

}  // namespace soil
