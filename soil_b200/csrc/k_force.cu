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
#include <cstdlib>
#include <cstring>

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

__global__ void __launch_bounds__(kBlock) k_seq_count(SeqArgs q, uint32_t* cnt, uint32_t* grp) {
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < q.ntotal;
         a += (uint64_t)gridDim.x * blockDim.x)
        seq_count_atom(q, a, cnt, grp);
}

__global__ void __launch_bounds__(kBlock) k_seq_fill(SeqArgs q, const uint32_t* grp_start,
                                                     uint32_t* seq, uint8_t* owner) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < q.nlocal;
         t += (uint64_t)gridDim.x * blockDim.x)
        seq_fill_root(q, t, grp_start, seq, owner);
}

void launch_seq_count(cudaStream_t st, const SeqArgs& q, uint32_t* cnt, uint32_t* grp) {
    if (q.ntotal == 0) return;
    note_launch();
    k_seq_count<<<grid_wave<k_seq_count>(q.ntotal), kBlock, 0, st>>>(q, cnt, grp);
}

void launch_seq_fill(cudaStream_t st, const SeqArgs& q, const uint32_t* grp_start, uint32_t* seq,
                     uint8_t* owner) {
    if (q.nlocal == 0) return;
    note_launch();
    k_seq_fill<<<grid_wave<k_seq_fill>(q.nlocal), kBlock, 0, st>>>(q, grp_start, seq, owner);
}

// ---- the warp-cooperative consumer, one launch --------------------------------

template <int U, bool FOLD>
__global__ void __launch_bounds__(kBlock, 4) k_force_seq(ForceArgs p) {
    __shared__ ForceSmem<U> sm;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint64_t ntiles = (p.q.nlocal + 31) / 32;
    for (uint64_t w = (uint64_t)blockIdx.x * kForceWarps + wib; w < ntiles;
         w += (uint64_t)gridDim.x * kForceWarps)
        force_tile<U, FOLD>(p.q, p.c, p.rev, w, sm, lane, wib);
}

// PK: partner records from the packed copy (p.q.pk / q.pk set).
template <bool FOLD, bool PK>
__global__ void __launch_bounds__(kBlock, 4) k_force_walk(ForceArgs p) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < p.q.nlocal;
         t += (uint64_t)gridDim.x * blockDim.x)
        force_walk_root<FOLD, PK>(p.q, p.c, p.rev, t);
}

template <bool FOLD, bool PK>
__global__ void __launch_bounds__(kBlock, 4) k_force_csr(ForceCsr q, AtomCols c, PlaneList rev) {
    pdl_wait();  // launched with pdl_launch
    // grid-stride over whole blocks of kBlock roots, so a block's order
    // permutes its own roots
    for (uint64_t b = (uint64_t)blockIdx.x * kBlock; b < q.nlocal; b += (uint64_t)gridDim.x * kBlock) {
        const uint64_t k = b + threadIdx.x;
        if (k < q.nlocal) force_csr_root<FOLD, PK>(q, c, rev, q.order ? q.order[k] : k);
    }
}

// Entries of root t's walk: its and its images' in-lists and its row.
__device__ __forceinline__ uint32_t csr_work(const ForceCsr& q, uint64_t t) {
    uint32_t n = q.offsets[t + 1] - q.offsets[t] + q.in_start[t + 1] - q.in_start[t];
    if (q.newton)
        for (uint32_t f = q.fold_start[t]; f < q.fold_start[t + 1]; ++f) {
            const uint64_t g = q.nlocal + q.fold_list[f];
            n += q.in_start[g + 1] - q.in_start[g];
        }
    return n;
}

// One block per kBlock roots: a bitonic sort of (work, index) keys in
// shared memory.
__global__ void __launch_bounds__(kBlock) k_root_order(ForceCsr q, uint32_t* order) {
    __shared__ uint64_t key[kBlock];
    const uint64_t b = (uint64_t)blockIdx.x * kBlock;
    const uint32_t i = threadIdx.x;
    const uint64_t t = b + i;
    const uint32_t work = t < q.nlocal ? min(csr_work(q, t), 0xffffu) : 0xffffffffu;
    key[i] = ((uint64_t)work << 32) | (uint32_t)i;
    __syncthreads();
    for (uint32_t size = 2; size <= kBlock; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            const uint32_t j = i ^ stride;
            if (j > i) {
                const uint64_t a = key[i], c = key[j];
                const bool up = (i & size) == 0;
                if ((a > c) == up) {
                    key[i] = c;
                    key[j] = a;
                }
            }
            __syncthreads();
        }
    if (t < q.nlocal) order[t] = (uint32_t)(b + (uint32_t)key[i]);
}

void launch_root_order(cudaStream_t st, const ForceCsr& q, uint32_t* order) {
    if (q.nlocal == 0) return;
    note_launch();
    k_root_order<<<(unsigned)((q.nlocal + kBlock - 1) / kBlock), kBlock, 0, st>>>(q, order);
}

void launch_force_csr(cudaStream_t st, const ForceCsr& q, const AtomCols& c, const PlaneList& rev,
                      bool fold) {
    if (q.nlocal == 0) return;
    note_launch();
    // one resident wave at <= 64 registers, striding over blocks of roots
    // (measured faster than one block per kBlock roots, and than 5 blocks per
    // SM at 48 registers, which spills; and faster than spreading a block's
    // roots and their images over its threads as one item list with the fold
    // after a barrier: 0.287 against 0.251 ms at C2)
    const unsigned full = 148u * 4u;
    const unsigned need = (unsigned)((q.nlocal + kBlock - 1) / kBlock);
    const unsigned grid = need < full ? need : full;
    if (q.pk) {
        if (fold) pdl_launch(k_force_csr<true, true>, grid, kBlock, 0, st, q, c, rev);
        else pdl_launch(k_force_csr<false, true>, grid, kBlock, 0, st, q, c, rev);
    } else {
        if (fold) pdl_launch(k_force_csr<true, false>, grid, kBlock, 0, st, q, c, rev);
        else pdl_launch(k_force_csr<false, false>, grid, kBlock, 0, st, q, c, rev);
    }
}

template <int U>
static void launch_tiles(cudaStream_t st, const ForceArgs& p, bool fold) {
    const uint64_t ntiles = (p.q.nlocal + 31) / 32;
    const uint64_t need = (ntiles + kForceWarps - 1) / kForceWarps;
    const uint64_t full = 148ull * 4ull;  // one resident wave, grid-stride over the tiles
    const unsigned grid = (unsigned)(need < full ? need : full);
    if (fold) k_force_seq<U, true><<<grid, kBlock, 0, st>>>(p);
    else k_force_seq<U, false><<<grid, kBlock, 0, st>>>(p);
}

// The consumer kernel (SOIL_FORCE: gather, csr, tiles4, tiles2, walk); read at
// each call so a host can compare them on one system.
int force_variant() {
    const char* env = std::getenv("SOIL_FORCE");
    if (!env) return kDefaultForce;
    if (!std::strcmp(env, "gather")) return SOIL_FORCE_GATHER;
    if (!std::strcmp(env, "tiles4")) return SOIL_FORCE_TILES4;
    if (!std::strcmp(env, "tiles2")) return SOIL_FORCE_TILES2;
    if (!std::strcmp(env, "walk")) return SOIL_FORCE_WALK;
    if (!std::strcmp(env, "csr")) return SOIL_FORCE_CSR;
    return kDefaultForce;
}

void launch_force_seq(cudaStream_t st, const ForceArgs& p, bool fold, int variant) {
    if (p.q.nlocal == 0) return;
    note_launch();
    if (variant == SOIL_FORCE_WALK) {
        const unsigned full = 148u * 4u;  // one resident wave at <= 64 registers
        const unsigned need = (unsigned)((p.q.nlocal + kBlock - 1) / kBlock);
        const unsigned grid = need < full ? need : full;
        if (p.q.pk) {
            if (fold) k_force_walk<true, true><<<grid, kBlock, 0, st>>>(p);
            else k_force_walk<false, true><<<grid, kBlock, 0, st>>>(p);
        } else {
            if (fold) k_force_walk<true, false><<<grid, kBlock, 0, st>>>(p);
            else k_force_walk<false, false><<<grid, kBlock, 0, st>>>(p);
        }
    } else if (variant == SOIL_FORCE_TILES2) {
        launch_tiles<2>(st, p, fold);
    } else {
        launch_tiles<4>(st, p, fold);
    }
}

}  // namespace soil
