// border_ops.cuh — warp-tile routines of the borders pass (chain categories,
// see k_ghost.cu), shared by the single-system and the batched kernels.
//
// A warp tile is 32 consecutive locals, one per lane.  Pass 1 stores the face
// bits and, per category, the tile's member count (counts[k * nw + w]; row
// kBorderCats holds all images of the tile).  After a per-category scan
// (offs, same layout), pass 2 ranks each member inside its tile with a ballot
// and writes its image, its send entry, its ghost root/chain and its root's
// fold program.  Every routine is called by all 32 lanes of a warp.
#pragma once

#include "block_scan.cuh"
#include "device_ops.cuh"

namespace soil {

__device__ __forceinline__ bool cat_member(const BorderCats& cats, uint32_t bits, int k) {
    return (bits & cats.need[k]) == cats.need[k];
}

__device__ __forceinline__ uint32_t warp_exclusive_sum(uint32_t v, uint32_t lane) {
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    return incl - v;
}

// Pass 1 for warp tile w: local r = 32 w + lane.
__device__ __forceinline__ void border_warp_counts(const AtomCols& c, uint64_t nlocal,
                                                   const Geom& geom, int triclinic,
                                                   const double* lo, const double* hi,
                                                   const BorderCats& cats, uint8_t* face,
                                                   uint32_t* counts, uint64_t nw, uint64_t w,
                                                   uint32_t lane) {
    const uint64_t r = w * 32 + lane;
    uint32_t bits = 0;
    if (r < nlocal) {
        bits = face_bits(c, geom, triclinic, lo, hi, r);
        face[r] = (uint8_t)bits;
    }
    uint32_t mine = 0, images = 0;
    // a category can have members only if the tile's faces cover its need:
    // the categories of the OR of its bits (uniform over the warp)
    const uint32_t any = __reduce_or_sync(0xffffffffu, bits);
    const uint32_t mine_cats = cats.member[bits];
    for (uint32_t cand = cats.member[any]; cand; cand &= cand - 1) {
        const int k = __ffs(cand) - 1;
        const uint32_t n = __popc(__ballot_sync(0xffffffffu, (mine_cats >> k) & 1u));
        if (lane == (uint32_t)k) mine = n;
        images += n;
    }
    if (lane < kBorderCats) counts[lane * nw + w] = mine;
    if (lane == kBorderCats) counts[kBorderCats * nw + w] = images;
}

// Per-dim border state in the format the host reads (bs[0..9]) from the
// category totals bs[kBorderTotals + k].
__device__ __forceinline__ void border_state_words(const BorderCats& cats, uint64_t nlocal,
                                                   uint32_t* bs) {
    bs[0] = (uint32_t)nlocal;
    for (int d = 0; d < 3; ++d) {
        uint32_t n[2] = {0, 0};
        for (int side = 0; side < 2; ++side) {
            const int s = 2 * d + side;
            for (int q = 0; q < cats.swap_ncat[s]; ++q)
                n[side] += bs[kBorderTotals + cats.swap_first[s] + q];
        }
        bs[4 + d] = n[0];
        bs[7 + d] = n[1];
        bs[d + 1] = bs[d] + n[0] + n[1];
    }
}

// Warp tiles per scan chunk: the category scans run one CTA per (category,
// chunk); chunk prefixes (cpre[k * nchunks + chunk]) are added back here.
constexpr uint64_t kScanChunk = 8192;

// Shared-memory scratch of one warp in pass 2: every lane's ghost index per
// category (indexed by category, so it must not live in registers) and the
// first ghost index of each swap.
struct BorderWarpSmem {
    uint32_t idx[kBorderCats][32];
    uint32_t recv[kNumSwaps];
};

// Pass 2 for warp tile w.  base_lane: on lane k < 26 the first ghost index of
// category k (nlocal + the totals of the categories before it).  offs holds
// offsets inside the tile's scan chunk; cpre (NULL: a single chunk) the
// chunks' prefixes.  sm: this warp's scratch.  host_bs (optional): the host's
// copy of bs, which gets the capacity word too.
__device__ __forceinline__ void border_warp_images(
    const AtomCols& c, uint64_t nlocal, uint64_t cap, const double (*shift)[3],
    const double (*vshift)[3], const BorderCats& cats, const uint8_t* face, const uint32_t* offs,
    const uint32_t* cpre, uint64_t nchunks, uint64_t nw, uint64_t w, uint32_t lane,
    uint32_t base_lane, uint32_t* bs, uint32_t* root, uint32_t* chain, uint32_t* const* send,
    uint32_t* fold_start, uint32_t* fold_list, BorderWarpSmem& sm, uint32_t* host_bs = nullptr) {
    const unsigned below = (1u << lane) - 1u;
    const uint64_t r = w * 32 + lane;
    const uint32_t bits = r < nlocal ? face[r] : 0u;
    const uint64_t cw = w / kScanChunk;
    const uint32_t any = __reduce_or_sync(0xffffffffu, bits);
    if (!any) {  // no images: empty fold programs
        const uint32_t fold0 =
            offs[kBorderCats * nw + w] + (cpre ? cpre[kBorderCats * nchunks + cw] : 0u);
        if (r < nlocal) fold_start[r] = fold0;
        if (r + 1 == nlocal) fold_start[nlocal] = fold0;
        return;
    }
    // lane k <= 26: offset of this tile's members of category k (k = 26: images)
    const uint32_t off_lane =
        lane <= (uint32_t)kBorderCats
            ? offs[lane * nw + w] + (cpre ? cpre[lane * nchunks + cw] : 0u)
            : 0u;
    const uint32_t fold0 = __shfl_sync(0xffffffffu, off_lane, kBorderCats);
    const uint32_t rv =
        __shfl_sync(0xffffffffu, base_lane, lane < (uint32_t)kNumSwaps ? cats.swap_first[lane] : 0);
    if (lane < (uint32_t)kNumSwaps) sm.recv[lane] = rv;
    const uint32_t mine_cats = cats.member[bits];
    const uint32_t own = __popc(mine_cats);  // images of this lane's root
    // only categories the tile's faces cover can have members (uniform over
    // the warp); only members read idx, and a member's parent category has
    // it as a member too
    for (uint32_t cand = cats.member[any]; cand; cand &= cand - 1) {
        const int k = __ffs(cand) - 1;
        const unsigned bal = __ballot_sync(0xffffffffu, (mine_cats >> k) & 1u);
        const uint32_t base = __shfl_sync(0xffffffffu, base_lane + off_lane, k);
        sm.idx[k][lane] = base + __popc(bal & below);
    }
    __syncwarp();
    const uint32_t fs = fold0 + warp_exclusive_sum(own, lane);
    if (r < nlocal) fold_start[r] = fs;
    if (r + 1 == nlocal) fold_start[nlocal] = fs + own;
    if (bits) {
        for (uint32_t mk = mine_cats; mk; mk &= mk - 1) {
            const int k = __ffs(mk) - 1;
            const uint32_t g = sm.idx[k][lane];
            if (g >= cap) {
                bs[10] = 1u;  // out of capacity: the host grows the arrays and repeats
                if (host_bs) host_bs[10] = 1u;
                continue;
            }
            const uint32_t parent =
                cats.parent[k] < 0 ? (uint32_t)r : sm.idx[cats.parent[k]][lane];
            write_image(c, shift, vshift, cats, k, g, r, parent, nlocal, root, chain);
            const int s = cats.swap_of[k];
            send[s][g - sm.recv[s]] = parent;
        }
        uint32_t j = fs;
        for (uint32_t mf = cats.member_fold[bits]; mf; mf &= mf - 1) {
            const int k = cats.fold[__ffs(mf) - 1];
            const uint32_t g = sm.idx[k][lane];
            if (g < cap && j < cap) fold_list[j] = g - (uint32_t)nlocal;
            ++j;
        }
    }
    __syncwarp();  // every lane is done with the scratch before the warp's next tile
}

}  // namespace soil
