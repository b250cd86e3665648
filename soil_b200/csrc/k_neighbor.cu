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
#include "border_ops.cuh"
#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

// Pass 1: one thread per local row (rows of a warp are neighbours in space, so
// their candidate records are shared through L1); the first K entries go to
// the row's slots, the length to rowcount.
template <bool UNIFORM, bool FP32>
__global__ void __launch_bounds__(kBlock) k_pairs_rows(PairParams p, uint32_t* rowcount,
                                                       uint32_t* slots, DevFlags* flags) {
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
                                                       const uint32_t* offsets, uint32_t* indices) {
    const Filter<UNIFORM, FP32> test(p);
    const uint32_t K = (uint32_t)p.row_slots;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < p.nlocal;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t cnt = rowcount[i];
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
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k0 + u < cnt) a[u] = src[k0 + u];
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

// Pass 1 with the warp's 32 rows tested together (FP64 filter; stencils of
// at most kPreRanges - 1 runs).  Each lane holds its row's ranges (as
// row_scan_pre: the own range, merged with a first run at +1 with newton,
// then the runs).  Range by range, the warp lays its rows' candidates end to
// end (row after row, each in slot order) and tests them 32 at a time, every
// lane busy: lane l takes item base + l, finds its row by a search over the
// rows' item offsets, and tests that row's record (from the row's lane)
// against the candidate's.  A row's accepted entries are appended in item
// order, so each row is the same sequence as row_scan gives: its own range,
// then the runs in stencil order, each in slot order.
template <bool UNIFORM>
__global__ void __launch_bounds__(kBlock) k_pairs_warp(PairParams p, uint32_t* rowcount,
                                                       uint32_t* slots, DevFlags* flags) {
    const Filter<UNIFORM, false> test(p);
    const uint32_t K = (uint32_t)p.row_slots;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t ntiles = (p.nlocal + 31) / 32;
    const uint64_t nwarps = (uint64_t)gridDim.x * (kBlock / 32);
    uint64_t n_cand = 0;
    for (uint64_t w = ((uint64_t)blockIdx.x * kBlock + threadIdx.x) / 32; w < ntiles; w += nwarps) {
        const uint64_t i = w * 32 + lane;
        const bool valid = i < p.nlocal;
        uint32_t my_cell = 0, mi = 0;
        double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
        uint32_t rm[kPreRanges], re[kPreRanges];
#pragma unroll
        for (int k = 0; k < kPreRanges; ++k) {
            rm[k] = 0;
            re[k] = 0;
        }
        if (valid) {
            my_cell = p.atom_cell[i];
            mi = p.atom_sorted_idx[i];
            pi = ld_rec(p.sp + mi);
            int first = 0;
            if (p.has_self) {
                uint64_t ce = (uint64_t)my_cell + 1;
                if (p.newton && p.nstencil > 0 && p.stencil[0] == 1 &&
                    ce + (uint64_t)p.stencil[1] <= p.ncells) {
                    ce += (uint64_t)p.stencil[1];
                    first = 1;
                }
                rm[0] = p.newton ? mi + 1 : p.bin_start[my_cell];
                re[0] = p.bin_start[ce];
            }
#pragma unroll
            for (int k = 1; k < kPreRanges; ++k) {
                const int s = first + k - 1;
                if (s < p.nstencil) {
                    const int64_t c0 = (int64_t)my_cell + p.stencil[2 * s];
                    const int64_t c1 = c0 + p.stencil[2 * s + 1];
                    if (c0 < 0 || c1 > (int64_t)p.ncells) {  // unreachable with the ghost layers
                        atomicOr(&flags->error, 1u);
                    } else {
                        rm[k] = p.bin_start[c0];
                        re[k] = p.bin_start[c1];
                    }
                }
            }
        }
        const bool skip_i = valid && p.has_self && !p.newton;  // i is in its own range
        uint32_t cnt = 0;
#pragma unroll
        for (int k = 0; k < kPreRanges; ++k) {
            const uint32_t L = re[k] - rm[k];
            n_cand += L;
            const uint32_t P = warp_exclusive_sum(L, lane);
            const uint32_t T = __shfl_sync(0xffffffffu, P + L, 31);
            const uint32_t m0 = rm[k];
            for (uint32_t base = 0; base < T; base += 32) {
                const uint32_t item = base + lane;
                const bool active = item < T;
                // the row of this item: the last lane whose offset is <= item
                uint32_t row = 0;
#pragma unroll
                for (uint32_t step = 16; step > 0; step >>= 1)
                    if (__shfl_sync(0xffffffffu, P, row + step) <= item) row += step;
                const uint32_t prow = __shfl_sync(0xffffffffu, P, row);
                const uint32_t slot = __shfl_sync(0xffffffffu, m0, row) + (item - prow);
                double4 prec;
                prec.x = __shfl_sync(0xffffffffu, pi.x, row);
                prec.y = __shfl_sync(0xffffffffu, pi.y, row);
                prec.z = __shfl_sync(0xffffffffu, pi.z, row);
                prec.w = __shfl_sync(0xffffffffu, pi.w, row);
                // without newton the own range holds the row's own atom: not a candidate
                const uint32_t mrow =
                    k == 0 ? __shfl_sync(0xffffffffu, skip_i ? mi : 0xffffffffu, row) : 0xffffffffu;
                bool ok = false;
                if (active && slot != mrow) ok = test.test64(prec, ld_rec(p.sp + slot));
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                // rank among this row's accepted items of the chunk
                const uint32_t row_lo = prow > base ? prow - base : 0u;
                const unsigned below = (1u << lane) - 1u;
                const unsigned row_below = below & ~((1u << row_lo) - 1u);
                const uint32_t pos = __shfl_sync(0xffffffffu, cnt, row) + __popc(bal & row_below);
                if (ok) {
                    const uint32_t a = p.sorted_atoms[slot];
                    if (p.in_count) atomicAdd(&p.in_count[a], 1u);
                    if (pos < K) slots[(w * 32 + row) * K + pos] = a;
                }
                // each row counts its accepted items of the chunk
                const int64_t lo = (int64_t)P - (int64_t)base, hi = lo + (int64_t)L;
                const uint32_t l0 = lo < 0 ? 0u : lo > 32 ? 32u : (uint32_t)lo;
                const uint32_t l1 = hi < 0 ? 0u : hi > 32 ? 32u : (uint32_t)hi;
                const unsigned mine = l1 > l0 ? (l1 - l0 == 32 ? 0xffffffffu
                                                               : ((1u << (l1 - l0)) - 1u) << l0)
                                              : 0u;
                cnt += __popc(bal & mine);
            }
        }
        if (valid) rowcount[i] = cnt;
        if (skip_i) n_cand -= 1;
    }
    __shared__ unsigned long long s_cand;
    if (threadIdx.x == 0) s_cand = 0;
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) n_cand += __shfl_down_sync(0xffffffffu, n_cand, o);
    if (lane == 0) atomicAdd(&s_cand, (unsigned long long)n_cand);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd((unsigned long long*)&flags->candidates, s_cand);
}

template <bool UNIFORM, bool FP32>
static void launch_pairs_t(cudaStream_t st, const PairParams& p, uint32_t* rowcount,
                           uint32_t* slots, const uint32_t* offsets, uint32_t* indices,
                           DevFlags* flags, bool fill) {
    note_launch();
    if (!fill && !FP32 && p.warp_rows && p.nstencil < kPreRanges)
        k_pairs_warp<UNIFORM><<<grid_wave<k_pairs_warp<UNIFORM>>(p.nlocal), kBlock, 0, st>>>(
            p, rowcount, slots, flags);
    else if (!fill)
        k_pairs_rows<UNIFORM, FP32><<<grid_wave<k_pairs_rows<UNIFORM, FP32>>(p.nlocal), kBlock, 0, st>>>(p, rowcount, slots,
                                                                            flags);
    else
        k_pairs_fill<UNIFORM, FP32><<<grid_wave<k_pairs_fill<UNIFORM, FP32>>(p.nlocal), kBlock, 0, st>>>(p, rowcount, slots,
                                                                            offsets, indices);
}

static void dispatch_pairs(cudaStream_t st, const PairParams& p, uint32_t* rowcount,
                           uint32_t* slots, const uint32_t* offsets, uint32_t* indices,
                           DevFlags* flags, bool fill) {
    const bool fp32 = p.filter == SOIL_FILTER_FP32_RECHECK;
    if (p.uniform) {
        if (fp32) launch_pairs_t<true, true>(st, p, rowcount, slots, offsets, indices, flags, fill);
        else launch_pairs_t<true, false>(st, p, rowcount, slots, offsets, indices, flags, fill);
    } else {
        if (fp32) launch_pairs_t<false, true>(st, p, rowcount, slots, offsets, indices, flags, fill);
        else launch_pairs_t<false, false>(st, p, rowcount, slots, offsets, indices, flags, fill);
    }
}

void launch_pair_count(cudaStream_t st, const PairParams& p, uint32_t* rowcount, uint32_t* slots,
                       DevFlags* flags) {
    if (p.nlocal == 0 || p.ncells == 0) return;
    dispatch_pairs(st, p, rowcount, slots, nullptr, nullptr, flags, false);
}

void launch_pair_fill(cudaStream_t st, const PairParams& p, const uint32_t* rowcount,
                      const uint32_t* slots, const uint32_t* offsets, uint32_t* indices) {
    if (p.nlocal == 0) return;
    dispatch_pairs(st, p, const_cast<uint32_t*>(rowcount), const_cast<uint32_t*>(slots), offsets,
                   indices, nullptr, true);
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
