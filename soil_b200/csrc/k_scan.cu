// k_scan.cu — device-wide exclusive scan of u32 counts (bin counts, row
// counts, ghost tile counts).  Three passes over tiles of 2048 items:
// tile sums -> one-CTA scan of the sums -> tile scans with the carry-in.
// 256 threads x 8 consecutive items per thread; warp shuffles inside a warp,
// shared memory across the 8 warps.
#include "block_scan.cuh"
#include "kernels.cuh"

namespace soil {

constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

__global__ void __launch_bounds__(kBlock) k_scan_reduce(const uint32_t* in, uint64_t n,
                                                        uint32_t* partial) {
    __shared__ uint32_t tot;
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) s += in[base + k];
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
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
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    uint32_t pre = block_exclusive_scan(s, &tot) + partial[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = partial[ntiles];
}

uint64_t scan_temp_words(uint64_t n) { return (n + kScanTile - 1) / kScanTile + 2; }

void exclusive_scan_u32(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n,
                        uint32_t* temp) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
        return;
    }
    note_launch();
    k_scan_reduce<<<(unsigned)ntiles, kBlock, 0, st>>>(in, n, temp);
    note_launch();
    k_scan_partials<<<1, kBlock, 0, st>>>(temp, ntiles);
    note_launch();
    k_scan_down<<<(unsigned)ntiles, kBlock, 0, st>>>(in, out, n, temp, ntiles);
}

}  // namespace soil
