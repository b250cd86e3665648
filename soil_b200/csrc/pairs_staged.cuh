// pairs_staged.cuh — device code of the staged pair count (one warp tile of
// 32 rows with its candidate records staged in shared memory by bulk copy),
// shared by the single-system kernel (k_pairs_staged.cu) and the batched one
// (k_batch.cu).  The method is described at the top of k_pairs_staged.cu.
#pragma once

#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {


constexpr int kStageWarps = 4;     // 128 threads per CTA
constexpr int kStageRecs = 256;    // staged records per warp
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// bytes (a multiple of 16) from global src to shared dst, both 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t it = 0; it < kWaitLimit; ++it)
        if (mbar_try(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ uint32_t warp_max(uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Row i (cell c) from the staged records, in the order of row_scan: the own
// cell's tail (newton) or the own cell without i, then the segments.
template <bool UNIFORM, bool FP32>
__device__ uint32_t row_scan_staged(const PairParams& p, const PairSegs& sg,
                                    const Filter<UNIFORM, FP32>& test, uint64_t i, uint32_t c,
                                    const unsigned char* recs, const uint32_t* lo,
                                    const uint32_t* base, uint32_t* out, uint32_t cap,
                                    uint32_t* rechk, uint32_t* cand) {
    constexpr int RS = FP32 ? 16 : 32;
    const uint32_t mi = p.atom_sorted_idx[i];
    const double4 pi = p.sp[mi];
    const float4 pif = FP32 ? p.spf[mi] : make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t cnt = 0;
    int s = -1;
    uint32_t m = 0, e = 0;
    bool own = false;
    for (;;) {
        while (m >= e) {  // open the next non-empty segment
            if (++s >= sg.n) return cnt;
            own = sg.own && s == 0;
            if (own) {
                e = p.bin_start[c + 1];
                m = p.newton ? mi + 1 : p.bin_start[c];
            } else {
                const uint32_t cc = (uint32_t)((int32_t)c + sg.off[s]);
                m = p.bin_start[cc];
                e = p.bin_start[cc + sg.len[s]];
                *cand += e - m;
            }
        }
        if (own) {  // own cell: i itself is not a candidate
            if (!p.newton && m == mi) {
                ++m;
                continue;
            }
            ++*cand;
        }
        const int r = sg.run[s];
        const unsigned char* rec = recs + (size_t)(base[r] + (m - lo[r])) * RS;
        bool ok;
        if (FP32) {
            ok = test.pass32(pif, *reinterpret_cast<const float4*>(rec));
            if (ok) {
                ++*rechk;
                ok = test.test64(pi, p.sp[m]);
            }
        } else {
            ok = test.test64(pi, *reinterpret_cast<const double4*>(rec));
        }
        if (ok) {
            const uint32_t a = p.sorted_atoms[m];
            if (p.in_count) atomicAdd(&p.in_count[a], 1u);
            if (cnt < cap) out[cnt] = a;
            ++cnt;
        }
        ++m;
    }
}

// One warp tile: rows [32 w, 32 w + 32) of a system.  Stages the tile's
// runs (when they fit) and writes every row's count and first K entries.
// recs: this warp's buffer (kStageRecs records of 32 B); s_lo / s_base: its
// kMaxPairSegs words each; phase: its mbarrier's parity.  Returns false when
// a staging wait ran out (the warp must stop).
template <bool UNIFORM, bool FP32>
__device__ bool staged_tile(const PairParams& p, const PairSegs& sg, uint64_t w,
                            unsigned char* recs, uint64_t* bar, uint32_t& phase, uint32_t* s_lo,
                            uint32_t* s_base, uint32_t* rowcount, uint32_t* slots,
                            DevFlags* flags, uint32_t& n_rechk, uint32_t& n_cand) {
    constexpr int RS = FP32 ? 16 : 32;
    const int lane = threadIdx.x & 31;
    const Filter<UNIFORM, FP32> test(p);
    const uint32_t K = (uint32_t)p.row_slots;
    const unsigned char* src = FP32 ? reinterpret_cast<const unsigned char*>(p.spf)
                                    : reinterpret_cast<const unsigned char*>(p.sp);
    const uint64_t i = w * 32 + lane;
    const bool valid = i < p.nlocal;
    const uint32_t c = valid ? p.atom_cell[i] : 0u;
    const uint32_t cA = warp_min(valid ? c : 0xffffffffu);
    const uint32_t cB = warp_max(valid ? c : 0u);
    // this tile's slot range of every staging run (lane r: run r)
    uint32_t lo = 0, n = 0;
    bool inside = true;
    if (lane < sg.nrun) {
        const int64_t a = (int64_t)cA + sg.roff[lane];
        const int64_t b = (int64_t)cB + sg.roff[lane] + sg.rlen[lane];
        if (a < 0 || b > (int64_t)p.ncells) {
            inside = false;
        } else {
            lo = p.bin_start[a];
            n = p.bin_start[b] - lo;
        }
    }
    uint32_t incl = n;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const bool staged = __all_sync(0xffffffffu, inside) && total <= (uint32_t)kStageRecs;
    if (staged && total > 0) {
        if (lane < sg.nrun) {
            s_lo[lane] = lo;
            s_base[lane] = incl - n;
        }
        __syncwarp();
        if (lane == 0) {
            // the buffer's previous contents were read through the generic
            // proxy; order those reads before the bulk copies overwrite it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, total * RS);
            for (int q = 0; q < sg.nrun; ++q) {
                const uint32_t b0 = s_base[q];
                const uint32_t b1 = q + 1 < sg.nrun ? s_base[q + 1] : total;
                if (b1 > b0)
                    bulk_g2s(recs + (size_t)b0 * RS, src + (size_t)s_lo[q] * RS, (b1 - b0) * RS,
                             bar);
            }
        }
        __syncwarp();
        // the whole warp takes the same branch
        if (!__all_sync(0xffffffffu, mbar_wait(bar, phase))) {
            if (lane == 0) atomicOr(&flags->error, SOIL_PAIRS_ERR_STAGING);
            mbar_wait(bar, phase);  // the copies in flight, bounded once more
            return false;
        }
        phase ^= 1u;
    }
    if (valid) {
        uint32_t cnt;
        if (staged)
            cnt = row_scan_staged<UNIFORM, FP32>(p, sg, test, i, c, recs, s_lo, s_base,
                                                 slots + i * K, K, &n_rechk, &n_cand);
        else
            cnt = row_scan<UNIFORM, FP32, true>(p, test, i, slots + i * K, K, &n_rechk, &n_cand,
                                                flags, p.in_count);
        rowcount[i] = cnt;
    }
    __syncwarp();  // every lane is done with the buffer and the ranges
    return true;
}

// Per-warp staging state at kernel start: lane 0 initialises the mbarrier.
__device__ __forceinline__ void staged_init(uint64_t* bar) {
    if ((threadIdx.x & 31) == 0) {
        mbar_init(bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
}

}  // namespace soil
