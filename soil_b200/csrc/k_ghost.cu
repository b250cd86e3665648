// k_ghost.cu — periodic / Lees–Edwards ghost images on one GPU.
//
// borders (comm.rs:682-860): for dim in x,y,z the lo swap (shift +L) then
// the hi swap (shift -L) scan the locals plus the ghosts of earlier dims in
// index order and append every atom inside the face slab.  On the device the
// whole pass is an order-preserving compaction over the locals alone (see
// "borders as chain categories" below), so ghost order, send lists and recv
// ranges equal the reference's.
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
#include <algorithm>
#include <vector>

#include "border_ops.cuh"
#include "kernels.cuh"

namespace soil {

// ---- borders as chain categories ---------------------------------------------
// A ghost made in dim d is tested again only in later dims, with coordinates
// its shift left unchanged (x shifts move x only, y shifts x and y, never z),
// so its face bits are its root local's.  Every ghost is therefore a root
// local plus a chain of swaps (at most one per dim, dims ascending), and the
// reference's ghost list is 26 chain categories in creation order — dim x:
// [x-] [x+]; dim y: for each side, [y] after every earlier chain
// (none, x-, x+); dim z likewise over the nine chains before it — each
// holding its roots in local index order.  A ghost's source (origin) is the
// same root's image one chain shorter; the reverse-comm fold of a root visits
// its images in a fixed category order (build_border_cats' key: per level
// the swap priority 4,5,2,3,0,1 -> 0..5, 7 past the chain's end).
namespace {
BorderCats build_border_cats() {
    BorderCats t{};
    struct Chain {
        int n;
        int sw[3];
    };
    std::vector<Chain> scan{{0, {0, 0, 0}}};  // chains scanned by the current dim
    std::vector<Chain> cats;
    for (int d = 0; d < 3; ++d) {
        std::vector<Chain> made;
        for (int side = 0; side < 2; ++side) {
            t.swap_first[2 * d + side] = (uint8_t)cats.size();
            for (const Chain& c : scan) {
                Chain n = c;
                n.sw[n.n++] = 2 * d + side;
                cats.push_back(n);
                made.push_back(n);
            }
            t.swap_ncat[2 * d + side] = (uint8_t)scan.size();
        }
        scan.insert(scan.end(), made.begin(), made.end());
    }
    auto key = [](const Chain& c) {
        uint32_t k = 0;
        for (int l = 0; l < 3; ++l) {
            const uint32_t pr = l < c.n ? (2u - (uint32_t)c.sw[l] / 2u) * 2u + ((uint32_t)c.sw[l] & 1u) : 7u;
            k = k * 8u + pr;
        }
        return k;
    };
    std::vector<int> order;
    for (int k = 0; k < kBorderCats; ++k) {
        const Chain& c = cats[k];
        t.len[k] = (uint8_t)c.n;
        uint8_t need = 0;
        for (int l = 0; l < c.n; ++l) {
            t.sw[k][l] = (uint8_t)c.sw[l];
            need |= (uint8_t)(1u << c.sw[l]);
        }
        t.need[k] = need;
        t.swap_of[k] = (uint8_t)c.sw[c.n - 1];
        t.parent[k] = -1;
        for (int q = 0; q < kBorderCats && c.n > 1; ++q)
            if (cats[q].n == c.n - 1 &&
                std::equal(cats[q].sw, cats[q].sw + cats[q].n, c.sw))
                t.parent[k] = (int8_t)q;
        order.push_back(k);
    }
    std::sort(order.begin(), order.end(), [&](int a, int b) { return key(cats[a]) < key(cats[b]); });
    for (int k = 0; k < kBorderCats; ++k) t.fold[k] = (uint8_t)order[k];
    return t;
}
}  // namespace

void finish_border_cats(BorderCats& t) {
    for (uint32_t bits = 0; bits < 64; ++bits) {
        uint32_t m = 0, mf = 0;
        for (int k = 0; k < kBorderCats; ++k)
            if ((bits & t.need[k]) == t.need[k]) m |= 1u << k;
        for (int f = 0; f < kBorderCats; ++f)
            if (m & (1u << t.fold[f])) mf |= 1u << f;
        t.member[bits] = m;
        t.member_fold[bits] = mf;
    }
}

const BorderCats& border_cats() {
    static const BorderCats t = [] {
        BorderCats c = build_border_cats();
        finish_border_cats(c);
        return c;
    }();
    return t;
}

BorderCats border_cats_masked(unsigned periodic_swaps) {
    BorderCats t = border_cats();
    for (int k = 0; k < kBorderCats; ++k)
        for (int q = 0; q < t.len[k]; ++q)
            if (!(periodic_swaps & (1u << t.sw[k][q]))) t.need[k] = 0x80;  // no face bit 7
    finish_border_cats(t);
    return t;
}

BorderPass border_pass(const BorderDim bds[3]) {
    BorderPass bp;
    bp.geom = bds[0].geom;
    bp.triclinic = bds[0].triclinic;
    for (int d = 0; d < 3; ++d) {
        bp.lo[d] = bds[d].thresh_lo;
        bp.hi[d] = bds[d].thresh_hi;
        for (int side = 0; side < 2; ++side)
            for (int q = 0; q < 3; ++q) {
                bp.shift[2 * d + side][q] = bds[d].shift[side][q];
                bp.vshift[2 * d + side][q] = bds[d].vshift[side][q];
            }
    }
    return bp;
}

// Pass 1, one warp per 32 locals: face bits, and per category the number of
// member roots of the warp (counts[k * nw + w]); counts[26 * nw + w] = all
// images of the warp's roots.
__global__ void __launch_bounds__(kBlock) k_border_faces(uint64_t nlocal, AtomCols c, BorderPass bp,
                                                         BorderCats cats, uint8_t* face,
                                                         uint32_t* counts, uint64_t nw) {
    pdl_wait();  // launched with pdl_launch
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; w < nw; w += nwarps)
        border_warp_counts(c, nlocal, bp.geom, bp.triclinic, bp.lo, bp.hi, cats, face, counts, nw,
                           w, lane);
}

// Pass 2: one CTA per (category or all images, chunk of kScanChunk warp
// tiles) scans the warp counts inside its chunk; ctot gets the chunk totals.
__global__ void __launch_bounds__(kBlock) k_border_cat_scan(const uint32_t* counts, uint32_t* offs,
                                                            uint64_t nw, uint32_t* ctot,
                                                            uint64_t nchunks) {
    pdl_wait();  // launched with pdl_launch
    const uint64_t k = blockIdx.x / nchunks, ch = blockIdx.x % nchunks;
    const uint64_t w0 = ch * kScanChunk;
    const uint64_t n = nw - w0 < kScanChunk ? nw - w0 : kScanChunk;
    const uint32_t total = cta_scan_array<8>(counts + k * nw + w0, offs + k * nw + w0, nullptr, n);
    if (threadIdx.x == 0) ctot[k * nchunks + ch] = total;
}

// Chunk totals -> exclusive chunk prefixes (in place) and category totals;
// clears the capacity word bs[10] that pass 3 may set.
__global__ void __launch_bounds__(kBlock) k_border_chunk_prefix(uint32_t* ctot, uint64_t nchunks,
                                                                uint32_t* bs, uint32_t* host_bs) {
    pdl_wait();  // launched with pdl_launch
    if (threadIdx.x == 0) {
        bs[10] = 0u;
        if (host_bs) host_bs[10] = 0u;
    }
    for (uint32_t k = threadIdx.x; k <= (uint32_t)kBorderCats; k += blockDim.x) {
        uint32_t acc = 0;
        for (uint64_t ch = 0; ch < nchunks; ++ch) {
            const uint32_t v = ctot[k * nchunks + ch];
            ctot[k * nchunks + ch] = acc;
            acc += v;
        }
        bs[kBorderTotals + k] = acc;
    }
}

// Pass 3, one warp per 32 locals: every image of the warp's roots at its
// final index, the swap send lists, ghost root/chain, and each root's fold
// program (its images in fold order).
__global__ void __launch_bounds__(kBlock) k_border_images(
    uint64_t nlocal, uint64_t cap, AtomCols c, BorderPass bp, BorderCats cats, const uint8_t* face,
    const uint32_t* offs, const uint32_t* cpre, uint64_t nchunks, uint64_t nw, uint32_t* bs,
    uint32_t* root, uint32_t* chain, SendPtrs send, uint32_t* fold_start, uint32_t* fold_list,
    uint32_t* host_bs) {
    pdl_wait();  // launched with pdl_launch
    __shared__ BorderWarpSmem sm[kBlock / 32];
    const uint32_t lane = threadIdx.x & 31u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        border_state_words(cats, nlocal, bs);
        if (host_bs)
            for (int k = 0; k < 10; ++k) host_bs[k] = bs[k];
    }
    // first ghost index of category `lane` (lanes below 26)
    const uint32_t tot = lane < kBorderCats ? bs[kBorderTotals + lane] : 0u;
    const uint32_t base_lane = (uint32_t)nlocal + warp_exclusive_sum(tot, lane);
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; w < nw; w += nwarps)
        border_warp_images(c, nlocal, cap, bp.shift, bp.vshift, cats, face, offs, cpre, nchunks,
                           nw, w, lane, base_lane, bs, root, chain, send.p, fold_start, fold_list,
                           sm[threadIdx.x / 32], host_bs);
}

void launch_borders(cudaStream_t st, uint64_t nlocal, uint64_t cap, const AtomCols& c,
                    const BorderCats& cats, const BorderPass& bp, uint8_t* face, uint32_t* counts,
                    uint32_t* offs, uint32_t* bs, uint32_t* ghost_root, uint32_t* ghost_chain,
                    const SendPtrs& send, uint32_t* fold_start, uint32_t* fold_list,
                    uint32_t* host_bs) {
    if (nlocal == 0) return;
    const uint64_t nw = (nlocal + 31) / 32;
    const uint64_t nchunks = (nw + kScanChunk - 1) / kScanChunk;
    uint32_t* ctot = counts + (kBorderCats + 1) * nw;  // chunk totals, then prefixes
    note_launch();
    pdl_launch(k_border_faces, grid_wave<k_border_faces>(nw * 32), kBlock, 0, st, nlocal, c, bp, cats, face,
                                                                          counts, nw);
    note_launch();
    pdl_launch(k_border_cat_scan, (unsigned)((kBorderCats + 1) * nchunks), kBlock, 0, st, counts, offs, nw,
                                                                                ctot, nchunks);
    note_launch();
    pdl_launch(k_border_chunk_prefix, 1, kBlock, 0, st, ctot, nchunks, bs, host_bs);
    note_launch();
    pdl_launch(k_border_images, grid_wave<k_border_images>(nw * 32), kBlock, 0, st, 
        nlocal, cap, c, bp, cats, face, offs, ctot, nchunks, nw, bs, ghost_root, ghost_chain, send,
        fold_start, fold_list, host_bs);
}

__global__ void __launch_bounds__(kBlock) k_forward(uint64_t nlocal, uint64_t nghost, AtomCols c,
                                                    const uint32_t* root, const uint32_t* chain,
                                                    SwapConst sc, PlaneList fwd, int zero_force) {
    pdl_wait();  // launched with pdl_launch
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
    pdl_launch(k_forward, grid_wave<k_forward>(nghost), kBlock, 0, st, nlocal, nghost, c, ghost_root, ghost_chain, sc,
                                                   pl, zero_force ? 1 : 0);
}

// ---- reverse comm as one fold per image tree ------------------------------
// The reference folds ghost forces swap by swap, last round first, lo before
// hi: target X receives, in order, its children through swaps 4, 5, 2, 3, 0, 1,
// each child already holding its own children's folds.  That is a post-order
// walk of each local atom's image tree with children ordered by that swap
// priority; the borders pass writes each root's images in that order (its
// fold program), and applying F[origin[g]] += F[g] along it reproduces every
// addition of the reference, intermediate ghosts included.
__global__ void __launch_bounds__(kBlock) k_reverse_fold(uint64_t nlocal, const uint32_t* start,
                                                         const uint32_t* list, AtomCols c,
                                                         PlaneList rev) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nlocal;
         t += (uint64_t)gridDim.x * blockDim.x)
        fold_root(c, nlocal, t, start, list, rev);
}

// Only the roots with images: after a border pass most locals have none, and
// a pass over all of them is a scan of fold_start for a few percent of work.
__global__ void __launch_bounds__(kBlock) k_reverse_fold_roots(uint64_t nlocal,
                                                               const uint32_t* count,
                                                               const uint32_t* roots,
                                                               const uint32_t* start,
                                                               const uint32_t* list, AtomCols c,
                                                               PlaneList rev) {
    const uint64_t n = *count;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < n;
         q += (uint64_t)gridDim.x * blockDim.x)
        fold_root(c, nlocal, roots[q], start, list, rev);
}

void launch_reverse_fold_roots(cudaStream_t st, uint64_t nlocal, uint64_t max_roots,
                               const uint32_t* count, const uint32_t* roots,
                               const uint32_t* start, const uint32_t* list, const AtomCols& c,
                               const int* rev_planes, int nrev) {
    if (max_roots == 0) return;
    PlaneList pl;
    pl.n = nrev;
    for (int k = 0; k < nrev; ++k) pl.idx[k] = rev_planes[k];
    note_launch();
    k_reverse_fold_roots<<<grid_wave<k_reverse_fold_roots>(max_roots), kBlock, 0, st>>>(nlocal, count, roots, start, list,
                                                                 c, pl);
}

__global__ void __launch_bounds__(kBlock) k_fold_root_flags(uint64_t nlocal,
                                                            const uint32_t* fold_start,
                                                            uint32_t* flag) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nlocal;
         t += (uint64_t)gridDim.x * blockDim.x)
        flag[t] = fold_start[t + 1] != fold_start[t] ? 1u : 0u;
}

void launch_fold_root_flags(cudaStream_t st, uint64_t nlocal, const uint32_t* fold_start,
                            uint32_t* flag) {
    if (nlocal == 0) return;
    note_launch();
    k_fold_root_flags<<<grid_wave<k_fold_root_flags>(nlocal), kBlock, 0, st>>>(nlocal, fold_start, flag);
}

void launch_reverse_fold(cudaStream_t st, uint64_t nlocal, const uint32_t* start,
                         const uint32_t* list, const AtomCols& c, const int* rev_planes, int nrev) {
    if (nlocal == 0) return;
    PlaneList pl;
    pl.n = nrev;
    for (int k = 0; k < nrev; ++k) pl.idx[k] = rev_planes[k];
    note_launch();
    k_reverse_fold<<<grid_wave<k_reverse_fold>(nlocal), kBlock, 0, st>>>(nlocal, start, list, c, pl);
}

}  // namespace soil
