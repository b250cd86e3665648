// k_scan.cu — device-wide exclusive scan of u32 counts (bin counts, row
// counts, ghost tile counts).  Three passes over tiles of 2048 items:
// tile sums -> one-CTA scan of the sums -> tile scans with the carry-in.
// 256 threads x 8 consecutive items per thread; warp shuffles inside a warp,
// shared memory across the 8 warps.
#include <atomic>
#include <cuda/atomic>

#include "block_scan.cuh"
#include "kernels.cuh"

namespace soil {

constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

// A thread's 8 consecutive items [base, base + 8) (zero past n): two 16-byte
// loads when the group is whole and aligned, else one by one.
__device__ __forceinline__ void load8(const uint32_t* in, uint64_t base, uint64_t n,
                                      uint32_t (&v)[kScanItems]) {
    if (base + kScanItems <= n && (reinterpret_cast<uintptr_t>(in + base) & 15u) == 0) {
        const uint4 a = *reinterpret_cast<const uint4*>(in + base);
        const uint4 b = *reinterpret_cast<const uint4*>(in + base + 4);
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        return;
    }
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = (base + k < n) ? in[base + k] : 0u;
}

// out[base + k] = pre + v[0] + ... + v[k - 1] for the items below n.
__device__ __forceinline__ void store8_scan(uint32_t* out, uint64_t base, uint64_t n,
                                            const uint32_t (&v)[kScanItems], uint32_t pre) {
    uint32_t o[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        o[k] = pre;
        pre += v[k];
    }
    if (base + kScanItems <= n && (reinterpret_cast<uintptr_t>(out + base) & 15u) == 0) {
        *reinterpret_cast<uint4*>(out + base) = make_uint4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<uint4*>(out + base + 4) = make_uint4(o[4], o[5], o[6], o[7]);
        return;
    }
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) out[base + k] = o[k];
}

// Up to two independent scans in one launch: blocks [0, tiles0) take tiles of
// scan 0, the rest tiles of scan 1 (each with its own partials).
struct ScanJobs {
    const uint32_t* in[2];
    uint32_t* out[2];
    uint64_t n[2];
    uint32_t* partial[2];
    uint64_t ntiles[2];
};

// This block's scan: its fields picked by selects (a parameter array indexed
// by a run-time value would be copied to local memory).
struct ScanJob {
    const uint32_t* in;
    uint32_t* out;
    uint64_t n;
    uint32_t* partial;
    uint64_t ntiles;
    uint64_t tile;  // this block's tile of it
};

__device__ __forceinline__ ScanJob scan_job(const ScanJobs& J) {
    const bool second = blockIdx.x >= J.ntiles[0];
    ScanJob s;
    s.in = second ? J.in[1] : J.in[0];
    s.out = second ? J.out[1] : J.out[0];
    s.n = second ? J.n[1] : J.n[0];
    s.partial = second ? J.partial[1] : J.partial[0];
    s.ntiles = second ? J.ntiles[1] : J.ntiles[0];
    s.tile = second ? blockIdx.x - J.ntiles[0] : blockIdx.x;
    return s;
}

__global__ void __launch_bounds__(kBlock) k_scan_reduce(ScanJobs J) {
    pdl_wait();  // launched with pdl_launch
    __shared__ uint32_t tot;
    const ScanJob q = scan_job(J);
    const uint64_t base = q.tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load8(q.in, base, q.n, v);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += v[k];
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) q.partial[q.tile] = tot;
}

// One CTA: exclusive scan of the tile sums in place, grand total to partial[ntiles].
__global__ void __launch_bounds__(kBlock) k_scan_partials(uint32_t* partial, uint64_t ntiles) {
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (uint64_t base = 0; base < ntiles; base += kScanTile) {
        const uint64_t b = base + (uint64_t)threadIdx.x * kScanItems;
        uint32_t v[kScanItems];
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            v[k] = (b + k < ntiles) ? partial[b + k] : 0;
            s += v[k];
        }
        uint32_t pre = block_exclusive_scan(s, &tot) + carry;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (b + k < ntiles) partial[b + k] = pre;
            pre += v[k];
        }
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[ntiles] = carry;
}

__global__ void __launch_bounds__(kBlock) k_scan_down(const uint32_t* in, uint32_t* out, uint64_t n,
                                                      const uint32_t* partial, uint64_t ntiles) {
    __shared__ uint32_t tot;
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load8(in, base, n, v);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += v[k];
    const uint32_t pre = block_exclusive_scan(s, &tot) + partial[blockIdx.x];
    store8_scan(out, base, n, v, pre);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = partial[ntiles];
}

// Pass 2 without the one-CTA pass over the tile sums: each CTA adds up the
// sums of the tiles before its own (at most kScanCarryTiles of them, read
// from L2), so the scan is two launches.  The last CTA writes out[n].
constexpr uint64_t kScanCarryTiles = 4096;

__global__ void __launch_bounds__(kBlock) k_scan_down_carry(ScanJobs J) {
    pdl_wait();  // launched with pdl_launch
    __shared__ uint32_t tot, s_carry;
    const ScanJob q = scan_job(J);
    const uint64_t t = q.tile, n = q.n;
    const uint32_t* partial = q.partial;
    const uint64_t base = t * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load8(q.in, base, n, v);
    uint32_t c = 0;  // this thread's share of the sums of tiles [0, t)
    for (uint64_t q = threadIdx.x; q < t; q += kBlock) c += partial[q];
    block_exclusive_scan(c, &tot);
    if (threadIdx.x == 0) s_carry = tot;
    __syncthreads();
    const uint32_t carry = s_carry;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += v[k];
    const uint32_t pre = block_exclusive_scan(s, &tot) + carry;
    store8_scan(q.out, base, n, v, pre);
    if (t + 1 == q.ntiles && threadIdx.x == 0) q.out[n] = carry + tot;
}

uint64_t scan_temp_words(uint64_t n) { return (n + kScanTile - 1) / kScanTile + 2; }

static ScanJobs one_job(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* temp) {
    ScanJobs J{};
    J.in[0] = in;
    J.out[0] = out;
    J.n[0] = n;
    J.partial[0] = temp;
    J.ntiles[0] = (n + kScanTile - 1) / kScanTile;
    return J;
}

void exclusive_scan_u32(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n,
                        uint32_t* temp) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
        return;
    }
    const ScanJobs J = one_job(in, out, n, temp);
    note_launch();
    pdl_launch(k_scan_reduce, (unsigned)ntiles, kBlock, 0, st, J);
    if (ntiles <= kScanCarryTiles) {
        note_launch();
        pdl_launch(k_scan_down_carry, (unsigned)ntiles, kBlock, 0, st, J);
        return;
    }
    note_launch();
    k_scan_partials<<<1, kBlock, 0, st>>>(temp, ntiles);
    note_launch();
    k_scan_down<<<(unsigned)ntiles, kBlock, 0, st>>>(in, out, n, temp, ntiles);
}

void exclusive_scan_u32_pair(cudaStream_t st, const uint32_t* in0, uint32_t* out0, uint64_t n0,
                             const uint32_t* in1, uint32_t* out1, uint64_t n1, uint32_t* temp) {
    const uint64_t t0 = (n0 + kScanTile - 1) / kScanTile, t1 = (n1 + kScanTile - 1) / kScanTile;
    if (t0 == 0 || t1 == 0 || t0 > kScanCarryTiles || t1 > kScanCarryTiles) {
        exclusive_scan_u32(st, in0, out0, n0, temp);
        exclusive_scan_u32(st, in1, out1, n1, temp + scan_temp_words(n0));
        return;
    }
    ScanJobs J = one_job(in0, out0, n0, temp);
    J.in[1] = in1;
    J.out[1] = out1;
    J.n[1] = n1;
    J.partial[1] = temp + scan_temp_words(n0);
    J.ntiles[1] = t1;
    note_launch();
    pdl_launch(k_scan_reduce, (unsigned)(t0 + t1), kBlock, 0, st, J);
    note_launch();
    pdl_launch(k_scan_down_carry, (unsigned)(t0 + t1), kBlock, 0, st, J);
}

// ---- single-pass scan (decoupled look-back) ---------------------------------
//
// One launch of ntiles CTAs.  Each CTA claims the next tile from an atomic
// counter (so every tile with a smaller number is held by a CTA that already
// runs), publishes its tile's sum, looks back over its predecessors'
// descriptors until it meets an inclusive prefix, publishes its own inclusive
// prefix and writes its tile.  A descriptor is 64 bits: the call's epoch (30
// bits), a status (1: tile sum, 2: inclusive prefix) and the value; the epoch
// makes descriptors of earlier calls read as not yet published, so nothing is
// cleared between calls.  The CTA that claims the last tile puts the counter
// back to zero.  Waits are bounded; one that runs out sets SOIL_SCAN_ERR in
// *err (when given) and counts the missing tiles as zero.

constexpr uint64_t kLookbackSpinLimit = 1ull << 22;
constexpr uint64_t kDescAgg = 1, kDescInc = 2;

__device__ __forceinline__ uint64_t desc_pack(uint32_t epoch, uint64_t status, uint32_t v) {
    return ((uint64_t)(epoch & 0x3fffffffu) << 34) | (status << 32) | v;
}

__global__ void __launch_bounds__(kBlock) k_scan_1p(const uint32_t* in, uint32_t* out, uint64_t n,
                                                    uint32_t* counter, uint64_t* desc,
                                                    uint32_t epoch, uint32_t* err) {
    __shared__ uint32_t s_tile, s_prefix, tot;
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (threadIdx.x == 0 && tile == ntiles - 1) atomicExch(counter, 0u);  // the last claim
    const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load8(in, base, n, v);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += v[k];
    uint32_t pre = block_exclusive_scan(s, &tot);
    const uint32_t agg = tot;
    const uint32_t ep = epoch & 0x3fffffffu;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t prefix = 0;
        if (tile == 0) {
            if (lane == 0)
                cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(desc[0]).store(
                    desc_pack(ep, kDescInc, agg), cuda::memory_order_release);
        } else {
            if (lane == 0)
                cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(desc[tile]).store(
                    desc_pack(ep, kDescAgg, agg), cuda::memory_order_release);
            int64_t look = (int64_t)tile - 1;
            for (;;) {
                const int64_t idx = look - lane;  // lane 0: the nearest predecessor
                uint64_t st = kDescInc;  // lanes past tile 0 take no part
                uint32_t val = 0;
                if (idx >= 0) {
                    cuda::atomic_ref<uint64_t, cuda::thread_scope_device> d(desc[idx]);
                    st = 0;
                    for (uint64_t spin = 0; spin < kLookbackSpinLimit; ++spin) {
                        const uint64_t x = d.load(cuda::memory_order_acquire);
                        if ((uint32_t)(x >> 34) == ep && ((x >> 32) & 3u)) {
                            st = (x >> 32) & 3u;
                            val = (uint32_t)x;
                            break;
                        }
                    }
                    if (st == 0) {
                        if (err) atomicOr(err, SOIL_SCAN_ERR);
                        st = kDescAgg;  // counted as zero
                    }
                }
                const unsigned inc = __ballot_sync(0xffffffffu, idx >= 0 && st == kDescInc);
                const int stop = inc ? __ffs(inc) - 1 : 31;
                uint32_t part = (lane <= stop && idx >= 0) ? val : 0u;
                for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
                prefix += part;
                if (inc || look - 32 < 0) break;
                look -= 32;
            }
            if (lane == 0)
                cuda::atomic_ref<uint64_t, cuda::thread_scope_device>(desc[tile]).store(
                    desc_pack(ep, kDescInc, prefix + agg), cuda::memory_order_release);
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    pre += s_prefix;
    store8_scan(out, base, n, v, pre);
    if (tile == ntiles - 1 && threadIdx.x == kBlock - 1) {
        uint32_t last = pre;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) last += v[k];
        out[n] = last;
    }
}

uint64_t scan1p_words(uint64_t n) { return 2 * ((n + kScanTile - 1) / kScanTile) + 4; }

static std::atomic<uint32_t> g_scan_epoch{1};

void exclusive_scan_1p(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n,
                       uint32_t* temp, uint32_t* err) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
        return;
    }
    const uint32_t epoch = g_scan_epoch.fetch_add(1, std::memory_order_relaxed);
    note_launch();
    k_scan_1p<<<(unsigned)ntiles, kBlock, 0, st>>>(in, out, n, temp,
                                                  reinterpret_cast<uint64_t*>(temp + 2), epoch,
                                                  err);
}

}  // namespace soil
