// k_neighbor.cu — half-list CSR build of bin_neighbor_list
// (neighbor.rs:1127-1319) and the transposed ("incoming") lists the
// deterministic force gather reads.
//
// Row order is the reference's: the self-cell tail (sorted slots after the
// atom's own slot), then every forward-stencil cell in stencil order, each
// cell in sorted (ascending index) order.
//
// Pass 1 (k_pairs_rows): one thread per local row scans its candidates in
// that order, keeps the first K accepted indices in fixed per-row slots and
// records the row length.  An exclusive scan of the lengths gives
// neighbor_offsets; pass 2 (k_pairs_fill) copies every row into place and
// re-derives, sequentially and in the same order, the rare rows longer than
// K.  (A warp-per-cell variant with ballot compaction was measured slower:
// one dependent-load chain per warp, no overlap across rows.)
//
// Candidates are read as one 32-byte record {x, y, z, cutoff} per sorted slot
// (sorted_pos of the reference plus the cutoff radius of the polydisperse
// test).  Filter: FP64 `fma(dx,dx,fma(dy,dy,dz*dz)) < cut^2` exactly as the
// reference, or (FP32 mode) a float test on grid-relative coordinates that
// only REJECTS candidates provably outside the cutoff — the margin eps bounds
// the float rounding of coordinates, differences and squares — followed by
// the exact FP64 test on the rest, so the lists are identical in both modes.
#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

// Pass 1: one thread per local row (rows of a warp are neighbours in space, so
// their candidate records are shared through L1); the first K entries go to
// the row's slots, the length to rowcount.
template <bool UNIFORM, bool FP32>
__global__ void __launch_bounds__(kBlock) k_pairs_rows(PairParams p, uint32_t* rowcount,
                                                       uint32_t* slots, DevFlags* flags) {
    pdl_wait();  // launched with pdl_launch
    const Filter<UNIFORM, FP32> test(p);
    const uint32_t K = (uint32_t)p.row_slots;
    uint32_t n_rechk = 0, n_cand32 = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < p.nlocal;
         i += (uint64_t)gridDim.x * blockDim.x)
        rowcount[i] = row_scan<UNIFORM, FP32, true>(p, test, i, slots + i * K, K, &n_rechk,
                                                    &n_cand32, flags, p.in_count);
    // the block's totals, then one atomic per counter and block (the FP64
    // filter rechecks nothing)
    __shared__ unsigned long long s_cand, s_rechk;
    if (threadIdx.x == 0) {
        s_cand = 0;
        s_rechk = 0;
    }
    __syncthreads();
    uint64_t n_cand = n_cand32;
    uint64_t r = n_rechk;
    for (int o = 16; o > 0; o >>= 1) {
        n_cand += __shfl_down_sync(0xffffffffu, n_cand, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_cand, (unsigned long long)n_cand);
        if (FP32) atomicAdd(&s_rechk, (unsigned long long)r);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd((unsigned long long*)&flags->candidates, s_cand);
        if (FP32) atomicAdd((unsigned long long*)&flags->rechecked, s_rechk);
    }
}

// Pass 2: rows into their CSR place; rows longer than K are re-derived.
template <bool UNIFORM, bool FP32>
__global__ void __launch_bounds__(kBlock) k_pairs_fill(PairParams p, const uint32_t* rowcount,
                                                       const uint32_t* slots,
                                                       const uint32_t* offsets, uint32_t* indices,
                                                       FillGuard g) {
    pdl_wait();  // launched with pdl_launch
    guard_publish(g);
    if (!guard_open(g)) return;
    const Filter<UNIFORM, FP32> test(p);
    const uint32_t K = (uint32_t)p.row_slots;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < p.nlocal;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t cnt = rowcount[i];
        // the row's first four slots, loaded with its length and offset (the
        // slots of a row are 16-byte aligned; past cnt they are unused)
        const uint4 head = *reinterpret_cast<const uint4*>(slots + i * K);
        uint32_t* out = indices + offsets[i];
        const bool slotted = cnt <= K;
        if (!slotted) {
            uint32_t rk = 0, cd = 0;
            row_scan<UNIFORM, FP32, true>(p, test, i, out, 0xffffffffu, &rk, &cd, nullptr);
        }
        // Four entries at a time, their loads, atomics and stores each issued
        // together: the row into its CSR place (from the slots) and (with the
        // transposed lists) row i into each partner's list, the counts going
        // back to 0.
        const uint32_t* src = slotted ? slots + i * K : out;
        for (uint32_t k0 = 0; k0 < cnt; k0 += 4) {
            uint32_t a[4], at[4];
            if (k0 == 0 && slotted) {
                a[0] = head.x;
                a[1] = head.y;
                a[2] = head.z;
                a[3] = head.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k0 + u < cnt) a[u] = src[k0 + u];
            }
            if (slotted) {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k0 + u < cnt) out[k0 + u] = a[u];
            }
            if (!p.in_list) continue;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k0 + u < cnt) at[u] = p.in_start[a[u]] + atomicSub(&p.in_count[a[u]], 1u) - 1u;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k0 + u < cnt) p.in_list[at[u]] = (uint32_t)i;
        }
    }
}

template <bool UNIFORM, bool FP32>
static void launch_pairs_t(cudaStream_t st, const PairParams& p, uint32_t* rowcount,
                           uint32_t* slots, const uint32_t* offsets, uint32_t* indices,
                           DevFlags* flags, const FillGuard* g) {
    note_launch();
    if (!g)
        pdl_launch(k_pairs_rows<UNIFORM, FP32>, grid_wave<k_pairs_rows<UNIFORM, FP32>>(p.nlocal), kBlock, 0, st, p, rowcount, slots,
                                                                            flags);
    else
        pdl_launch(k_pairs_fill<UNIFORM, FP32>, grid_wave<k_pairs_fill<UNIFORM, FP32>>(p.nlocal), kBlock, 0, st, p, rowcount, slots,
                                                                            offsets, indices, *g);
}

// g == nullptr: pass 1; else pass 2 under guard *g
static void dispatch_pairs(cudaStream_t st, const PairParams& p, uint32_t* rowcount,
                           uint32_t* slots, const uint32_t* offsets, uint32_t* indices,
                           DevFlags* flags, const FillGuard* g) {
    const bool fp32 = p.filter == SOIL_FILTER_FP32_RECHECK;
    if (p.uniform) {
        if (fp32) launch_pairs_t<true, true>(st, p, rowcount, slots, offsets, indices, flags, g);
        else launch_pairs_t<true, false>(st, p, rowcount, slots, offsets, indices, flags, g);
    } else {
        if (fp32) launch_pairs_t<false, true>(st, p, rowcount, slots, offsets, indices, flags, g);
        else launch_pairs_t<false, false>(st, p, rowcount, slots, offsets, indices, flags, g);
    }
}

void launch_pair_count(cudaStream_t st, const PairParams& p, uint32_t* rowcount, uint32_t* slots,
                       DevFlags* flags) {
    if (p.nlocal == 0 || p.ncells == 0) return;
    dispatch_pairs(st, p, rowcount, slots, nullptr, nullptr, flags, nullptr);
}

void launch_pair_fill(cudaStream_t st, const PairParams& p, const uint32_t* rowcount,
                      const uint32_t* slots, const uint32_t* offsets, uint32_t* indices,
                      const FillGuard& g) {
    if (p.nlocal == 0) return;
    dispatch_pairs(st, p, const_cast<uint32_t*>(rowcount), const_cast<uint32_t*>(slots), offsets,
                   indices, nullptr, &g);
}

__global__ void __launch_bounds__(kBlock) k_in_count(uint64_t nlocal, const uint32_t* offsets,
                                                     const uint32_t* indices, uint32_t* incount) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlocal;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (uint32_t q = offsets[i]; q < offsets[i + 1]; ++q) atomicAdd(&incount[indices[q]], 1u);
}

void launch_in_count(cudaStream_t st, uint64_t nlocal, const uint32_t* offsets,
                     const uint32_t* indices, uint32_t* incount) {
    if (nlocal == 0) return;
    note_launch();
    k_in_count<<<grid_wave<k_in_count>(nlocal), kBlock, 0, st>>>(nlocal, offsets, indices, incount);
}

__global__ void __launch_bounds__(kBlock) k_in_scatter(uint64_t nlocal, const uint32_t* offsets,
                                                       const uint32_t* indices, uint32_t* cursor,
                                                       uint32_t* in_list) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlocal;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (uint32_t q = offsets[i]; q < offsets[i + 1]; ++q)
            in_list[atomicAdd(&cursor[indices[q]], 1u)] = (uint32_t)i;
}

void launch_in_scatter(cudaStream_t st, uint64_t nlocal, const uint32_t* offsets,
                       const uint32_t* indices, uint32_t* cursor, uint32_t* in_list) {
    if (nlocal == 0) return;
    note_launch();
    k_in_scatter<<<grid_wave<k_in_scatter>(nlocal), kBlock, 0, st>>>(nlocal, offsets, indices, cursor, in_list);
}

}  // namespace soil
