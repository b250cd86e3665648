// k_ghost.cu — periodic / Lees–Edwards ghost images on one GPU.
//
// borders (comm.rs:682-860): for dim in x,y,z the lo swap (shift +L) then
// the hi swap (shift -L) scan the locals plus the ghosts of earlier dims in
// index order and append every atom inside the face slab.  The device version
// is an order-preserving stream compaction: per 512-atom tile count the lo
// and hi selections (storing each atom's face flags), scan the tile counts,
// then each tile ranks its flags with a CTA scan and writes the ghosts at
// their final slots — so ghost order, send lists and recv ranges equal the
// reference's.
//
// forward_comm (comm.rs:400-432): the reference packs pos+offset from the
// source (a local or an earlier ghost) swap by swap.  Every ghost therefore
// equals its root local atom plus the offsets of its swap chain, added in
// chain order; borders records (root, chain) so one kernel refreshes all
// ghosts with the exact same additions.
//
// reverse_send_force (comm.rs:938-1024): swaps are folded last to first,
// lo before hi, F[send[k]] += F[recv_start+k].  Per local atom that is a
// post-order walk of its image tree, done by one thread (see below).
#include "block_scan.cuh"
#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

constexpr int kBorderItems = kBorderTile / kBlock;

// Border state shared by the kernels of one borders pass (device memory):
//   bs[0..3]   scan_end of dim d (bs[0] = nlocal; bs[d+1] = bs[d] + lo_d + hi_d)
//   bs[4..6]   lo totals, bs[7..9] hi totals, bs[10] overflow flag
__global__ void __launch_bounds__(kBlock) k_border_count(uint32_t* bs, uint64_t cap, AtomCols c,
                                                         BorderDim bd, uint8_t* face,
                                                         uint32_t* tile_lo, uint32_t* tile_hi) {
    __shared__ uint32_t tot;
    const uint64_t scan_end = bs[bd.dim] < cap ? bs[bd.dim] : cap;  // a short pass is redone
    if ((uint64_t)blockIdx.x * kBorderTile >= scan_end) {  // tile past the scan range (uniform)
        if (threadIdx.x == 0) {
            tile_lo[blockIdx.x] = 0u;
            tile_hi[blockIdx.x] = 0u;
        }
        return;
    }
    const uint64_t base = (uint64_t)blockIdx.x * kBorderTile + (uint64_t)threadIdx.x * kBorderItems;
    uint32_t nlo = 0, nhi = 0;
    for (int k = 0; k < kBorderItems; ++k) {
        const uint64_t i = base + k;
        if (i >= scan_end) break;
        bool lo, hi;
        border_flags(c, bd, i, lo, hi);
        face[i] = (uint8_t)((lo ? 1 : 0) | (hi ? 2 : 0));
        nlo += lo;
        nhi += hi;
    }
    block_exclusive_scan(nlo, &tot);
    if (threadIdx.x == 0) tile_lo[blockIdx.x] = tot;
    block_exclusive_scan(nhi, &tot);
    if (threadIdx.x == 0) tile_hi[blockIdx.x] = tot;
}

// One CTA: exclusive scans of the lo and hi tile counts, the dim's totals and
// the next dim's scan_end.
__global__ void __launch_bounds__(kBlock) k_border_scan(uint32_t* bs, int dim, uint32_t ntiles,
                                                        const uint32_t* tile_lo,
                                                        const uint32_t* tile_hi, uint32_t* off_lo,
                                                        uint32_t* off_hi) {
    const uint32_t nlo = cta_scan_array<8>(tile_lo, off_lo, nullptr, ntiles);
    const uint32_t nhi = cta_scan_array<8>(tile_hi, off_hi, nullptr, ntiles);
    if (threadIdx.x == 0) {
        bs[4 + dim] = nlo;
        bs[7 + dim] = nhi;
        bs[dim + 1] = bs[dim] + nlo + nhi;
    }
}

__global__ void __launch_bounds__(kBlock) k_border_scatter(
    uint32_t* bs, uint64_t nlocal, uint64_t cap, AtomCols c, BorderDim bd, const uint8_t* face,
    const uint32_t* tile_cnt_lo, const uint32_t* tile_cnt_hi,
    const uint32_t* tile_off_lo, const uint32_t* tile_off_hi, uint32_t* send_lo,
    uint32_t* send_hi, uint32_t* root, uint32_t* chain) {
    __shared__ uint32_t tot;
    // nothing selected in this tile (counts of the count pass; uniform)
    if (tile_cnt_lo[blockIdx.x] == 0u && tile_cnt_hi[blockIdx.x] == 0u) return;
    const uint64_t scan_end = bs[bd.dim] < cap ? bs[bd.dim] : cap;
    const uint64_t recv_lo = bs[bd.dim];
    const uint64_t recv_hi = scan_end + bs[4 + bd.dim];
    const uint64_t base = (uint64_t)blockIdx.x * kBorderTile + (uint64_t)threadIdx.x * kBorderItems;
    uint32_t flo = 0, fhi = 0;  // bit k: item k selected
    for (int k = 0; k < kBorderItems; ++k) {
        const uint64_t i = base + k;
        if (i >= scan_end) break;
        const uint32_t f = face[i];
        flo |= (f & 1u) << k;
        fhi |= ((f >> 1) & 1u) << k;
    }
    uint32_t rlo = block_exclusive_scan(__popc(flo), &tot) + tile_off_lo[blockIdx.x];
    uint32_t rhi = block_exclusive_scan(__popc(fhi), &tot) + tile_off_hi[blockIdx.x];
    for (int k = 0; k < kBorderItems; ++k) {
        const uint64_t i = base + k;
        if ((flo >> k) & 1u) {
            if (recv_lo + rlo < cap) {
                write_ghost(c, recv_lo + rlo, i, bd.shift[0], bd.vshift[0], bd.swap_id[0], nlocal,
                            root, chain);
                send_lo[rlo] = (uint32_t)i;
            } else {
                bs[10] = 1u;  // out of capacity: the host grows the arrays and repeats borders
            }
            ++rlo;
        }
        if ((fhi >> k) & 1u) {
            if (recv_hi + rhi < cap) {
                write_ghost(c, recv_hi + rhi, i, bd.shift[1], bd.vshift[1], bd.swap_id[1], nlocal,
                            root, chain);
                send_hi[rhi] = (uint32_t)i;
            } else {
                bs[10] = 1u;
            }
            ++rhi;
        }
    }
}

// One dim of borders: count, scan, scatter (no host synchronisation).
void launch_border_dim(cudaStream_t st, uint32_t* bs, uint64_t nlocal, uint64_t cap,
                       const AtomCols& c, const BorderDim& bd, uint32_t max_tiles,
                       uint8_t* face_flags, uint32_t* tile_lo, uint32_t* tile_hi,
                       uint32_t* tile_off_lo, uint32_t* tile_off_hi, uint32_t* send_lo,
                       uint32_t* send_hi, uint32_t* ghost_root, uint32_t* ghost_chain) {
    if (max_tiles == 0) return;
    note_launch();
    k_border_count<<<max_tiles, kBlock, 0, st>>>(bs, cap, c, bd, face_flags, tile_lo, tile_hi);
    note_launch();
    k_border_scan<<<1, kBlock, 0, st>>>(bs, bd.dim, max_tiles, tile_lo, tile_hi, tile_off_lo,
                                        tile_off_hi);
    note_launch();
    k_border_scatter<<<max_tiles, kBlock, 0, st>>>(bs, nlocal, cap, c, bd, face_flags, tile_lo,
                                                   tile_hi, tile_off_lo, tile_off_hi, send_lo,
                                                   send_hi, ghost_root, ghost_chain);
}

__global__ void __launch_bounds__(kBlock) k_forward(uint64_t nlocal, uint64_t nghost, AtomCols c,
                                                    const uint32_t* root, const uint32_t* chain,
                                                    SwapConst sc, PlaneList fwd, int zero_force) {
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nghost;
         gi += (uint64_t)gridDim.x * blockDim.x)
        forward_ghost(c, nlocal, gi, root, chain, sc, fwd, zero_force != 0);
}

void launch_forward(cudaStream_t st, uint64_t nlocal, uint64_t nghost, const AtomCols& c,
                    const uint32_t* ghost_root, const uint32_t* ghost_chain, const SwapConst& sc,
                    const int* fwd_planes, int nfwd, bool zero_force) {
    if (nghost == 0) return;
    PlaneList pl;
    pl.n = nfwd;
    for (int k = 0; k < nfwd; ++k) pl.idx[k] = fwd_planes[k];
    note_launch();
    k_forward<<<grid_for(nghost), kBlock, 0, st>>>(nlocal, nghost, c, ghost_root, ghost_chain, sc,
                                                   pl, zero_force ? 1 : 0);
}

// ---- reverse comm as one fold per image tree ------------------------------
// The reference folds ghost forces swap by swap, last round first, lo before
// hi: target X receives, in order, its children through swaps 4, 5, 2, 3, 0, 1,
// each child already holding its own children's folds.  That is a post-order
// walk of each local atom's image tree with children ordered by that swap
// priority, so sorting a root's ghosts by a key built from their swap chains
// (priority per level, 7 past the end) and applying F[origin[g]] += F[g] in
// key order reproduces every addition of the reference, intermediate ghosts
// included.
__global__ void __launch_bounds__(kBlock) k_fold_count(uint64_t nghost, const uint32_t* root,
                                                       uint32_t* counts) {
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nghost;
         gi += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&counts[root[gi]], 1u);
}

__global__ void __launch_bounds__(kBlock) k_fold_scatter(uint64_t nghost, const uint32_t* root,
                                                         uint32_t* cursor, uint32_t* list) {
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nghost;
         gi += (uint64_t)gridDim.x * blockDim.x)
        list[atomicAdd(&cursor[root[gi]], 1u)] = (uint32_t)gi;
}

// per root: ghosts in post-order (key), ties impossible (one ghost per chain)
__global__ void __launch_bounds__(kBlock) k_fold_order(uint64_t nlocal, const uint32_t* start,
                                                       uint32_t* list, const uint32_t* chain) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nlocal;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = start[t], e = start[t + 1];
        for (uint32_t k = b + 1; k < e; ++k) {
            const uint32_t v = list[k];
            const uint32_t kv = fold_key(chain[v]);
            uint32_t j = k;
            while (j > b && fold_key(chain[list[j - 1]]) > kv) {
                list[j] = list[j - 1];
                --j;
            }
            list[j] = v;
        }
    }
}

void launch_fold_build(cudaStream_t st, uint64_t nlocal, uint64_t nghost,
                       const uint32_t* ghost_root, const uint32_t* ghost_chain, uint32_t* counts,
                       uint32_t* start, uint32_t* cursor, uint32_t* list, uint32_t* scan_tmp) {
    cudaMemsetAsync(counts, 0, nlocal * sizeof(uint32_t), st);
    if (nghost) {
        note_launch();
        k_fold_count<<<grid_for(nghost), kBlock, 0, st>>>(nghost, ghost_root, counts);
    }
    exclusive_scan_u32(st, counts, start, nlocal, scan_tmp);
    if (nghost == 0) return;
    cudaMemcpyAsync(cursor, start, nlocal * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    note_launch();
    k_fold_scatter<<<grid_for(nghost), kBlock, 0, st>>>(nghost, ghost_root, cursor, list);
    note_launch();
    k_fold_order<<<grid_for(nlocal), kBlock, 0, st>>>(nlocal, start, list, ghost_chain);
}

__global__ void __launch_bounds__(kBlock) k_reverse_fold(uint64_t nlocal, const uint32_t* start,
                                                         const uint32_t* list, AtomCols c,
                                                         PlaneList rev) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nlocal;
         t += (uint64_t)gridDim.x * blockDim.x)
        fold_root(c, nlocal, t, start, list, rev);
}

void launch_reverse_fold(cudaStream_t st, uint64_t nlocal, const uint32_t* start,
                         const uint32_t* list, const AtomCols& c, const int* rev_planes, int nrev) {
    if (nlocal == 0) return;
    PlaneList pl;
    pl.n = nrev;
    for (int k = 0; k < nrev; ++k) pl.idx[k] = rev_planes[k];
    note_launch();
    k_reverse_fold<<<grid_for(nlocal), kBlock, 0, st>>>(nlocal, start, list, c, pl);
}

}  // namespace soil
