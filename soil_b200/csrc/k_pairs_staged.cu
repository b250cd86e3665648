// k_pairs_staged.cu — the pair-count pass of bin_neighbor_list
// (crates/soil_core/src/neighbor.rs:1127-1319) with the candidate records
// staged in shared memory by bulk copy.
//
// A row's candidates are its own cell's tail and its stencil cells in
// stencil order.  The stencil offsets ascend, and a run of consecutive
// offsets is a run of consecutive cells, i.e. one contiguous range of sorted
// slots (PairSegs; segments of consecutive cells merge into staging runs).
// For a warp tile of 32 rows whose cells lie in [cA, cB], run r of every row
// lies inside the slot range [bin_start[cA + roff_r],
// bin_start[cB + roff_r + rlen_r]): lane 0 stages each
// of those ranges of the sorted records (sp, 32 B {x, y, z, cut}, or in FP32
// mode spf, 16 B) into the warp's shared buffer with cp.async.bulk on one
// mbarrier, from this GPU's own memory, and every lane then scans its row
// from shared memory in the reference's order (own cell, then the segments),
// writing the first K accepted indices to its row slots exactly as
// k_pairs_rows does.  Tiles whose ranges do not fit the buffer scan from
// global memory (row_scan).
//
// Waits on the mbarrier are bounded: a wait that runs out sets
// SOIL_PAIRS_ERR_STAGING in flags->error, waits (bounded) once more for the
// copies in flight, and ends the warp; the host turns the flag into an error.
#include "device_ops.cuh"
#include "kernels.cuh"
#include "pairs_staged.cuh"

namespace soil {

namespace {

template <bool UNIFORM, bool FP32>
__global__ void __launch_bounds__(kStageWarps * 32)
    k_pairs_staged(PairParams p, PairSegs sg, uint32_t* rowcount, uint32_t* slots,
                   DevFlags* flags) {
    constexpr int RS = FP32 ? 16 : 32;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint32_t s_lo[kStageWarps][kMaxPairSegs];
    __shared__ uint32_t s_base[kStageWarps][kMaxPairSegs];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char* recs = smem_raw + (size_t)wib * kStageRecs * RS;
    uint64_t* bar =
        reinterpret_cast<uint64_t*>(smem_raw + (size_t)kStageWarps * kStageRecs * RS) + wib;
    staged_init(bar);
    uint32_t phase = 0, n_rechk = 0, n_cand = 0;
    const uint64_t ntiles = (p.nlocal + 31) / 32;
    for (uint64_t w = (uint64_t)blockIdx.x * kStageWarps + wib; w < ntiles;
         w += (uint64_t)gridDim.x * kStageWarps)
        if (!staged_tile<UNIFORM, FP32>(p, sg, w, recs, bar, phase, s_lo[wib], s_base[wib],
                                        rowcount, slots, flags, n_rechk, n_cand))
            return;
    uint64_t nc = n_cand, r = n_rechk;
    for (int o = 16; o > 0; o >>= 1) {
        nc += __shfl_down_sync(0xffffffffu, nc, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
    }
    if (lane == 0) {
        atomicAdd((unsigned long long*)&flags->candidates, (unsigned long long)nc);
        atomicAdd((unsigned long long*)&flags->rechecked, (unsigned long long)r);
    }
}
template <bool UNIFORM, bool FP32>
void launch_staged_t(cudaStream_t st, const PairParams& p, const PairSegs& sg, uint32_t* rowcount,
                     uint32_t* slots, DevFlags* flags) {
    constexpr int RS = FP32 ? 16 : 32;
    const size_t smem = (size_t)kStageWarps * kStageRecs * RS + kStageWarps * sizeof(uint64_t);
    const uint64_t ntiles = (p.nlocal + 31) / 32;
    uint64_t blocks = (ntiles + kStageWarps - 1) / kStageWarps;
    const uint64_t cap = 148ull * 8ull;
    if (blocks > cap) blocks = cap;
    note_launch();
    k_pairs_staged<UNIFORM, FP32>
        <<<(unsigned)blocks, kStageWarps * 32, smem, st>>>(p, sg, rowcount, slots, flags);
}

}  // namespace

void launch_pair_count_staged(cudaStream_t st, const PairParams& p, const PairSegs& sg,
                              uint32_t* rowcount, uint32_t* slots, DevFlags* flags) {
    if (p.nlocal == 0 || p.ncells == 0) return;
    const bool fp32 = p.filter == SOIL_FILTER_FP32_RECHECK;
    if (p.uniform) {
        if (fp32) launch_staged_t<true, true>(st, p, sg, rowcount, slots, flags);
        else launch_staged_t<true, false>(st, p, sg, rowcount, slots, flags);
    } else {
        if (fp32) launch_staged_t<false, true>(st, p, sg, rowcount, slots, flags);
        else launch_staged_t<false, false>(st, p, sg, rowcount, slots, flags);
    }
}

}  // namespace soil
