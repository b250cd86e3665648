// block_scan.cuh — CTA-wide exclusive scan of one u32 per thread (kBlock threads).
#pragma once

#include "soil_internal.cuh"

namespace soil {

// Exclusive block scan of one value per thread; returns the prefix of this
// thread and writes the block total to *total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_tot[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kBlock / 32 ? warp_tot[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kBlock / 32) warp_tot[lane] = wi - w;  // exclusive warp offsets
        if (lane == kBlock / 32 - 1) *total = wi;
    }
    __syncthreads();
    const uint32_t res = warp_tot[warp] + inc - v;
    __syncthreads();
    return res;
}

// One CTA scans n values: out[t] (and out2[t] when given) = exclusive prefix
// of in over [0, n); returns the total.  ITEMS consecutive values per thread
// per pass, so a pass covers kBlock * ITEMS values.
template <int ITEMS>
__device__ __forceinline__ uint32_t cta_scan_array(const uint32_t* in, uint32_t* out,
                                                   uint32_t* out2, uint64_t n) {
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (uint64_t b0 = 0; b0 < n; b0 += (uint64_t)kBlock * ITEMS) {
        const uint64_t t0 = b0 + (uint64_t)threadIdx.x * ITEMS;
        uint32_t v[ITEMS];
        uint32_t sum = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            v[j] = t0 + j < n ? in[t0 + j] : 0u;
            sum += v[j];
        }
        uint32_t run = block_exclusive_scan(sum, &tot) + carry;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (t0 + j < n) {
                out[t0 + j] = run;
                if (out2) out2[t0 + j] = run;
            }
            run += v[j];
        }
        carry += tot;
        __syncthreads();
    }
    return carry;
}

}  // namespace soil
