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

}  // namespace soil
