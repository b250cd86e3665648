// k_batch.cu — segmented kernels of the batched engine (see batch.cuh).
//
// Three launch shapes:
//   element spans   blocks walk the flattened element range in chunks of
//                   kBlock * kSpanItems, locate the chunk's segment once and
//                   advance per element (boxes hold hundreds of atoms or more);
//   segment per CTA exclusive scans, one CTA per box;
//   tile spans      border tiles, one CTA per tile (the tile's CTA-wide scan
//                   ranks its ghosts in order).
// Every element calls the same device function as the single-system kernels.
#include "batch.cuh"
#include "block_scan.cuh"
#include "border_ops.cuh"
#include "force_ops.cuh"
#include "pairs_staged.cuh"
#include "sys_internal.cuh"

namespace soil {

constexpr int kSpanItems = 4;

// Segment holding flattened element g (the last segment whose start is <= g),
// found by the 32 lanes of one warp together: each level probes 32 evenly
// spaced starts, so 4,096 segments take three dependent loads.  Call with all
// 32 lanes of the warp; every lane returns the answer.
__device__ __forceinline__ uint32_t seg_of_warp(const Span& sp, uint64_t g) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lo = 0, hi = sp.nseg;  // start[lo] <= g < start[hi]
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + lane * step;
        const bool ok = idx < hi && sp.start[idx] <= g;
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        const uint32_t last = 31u - (uint32_t)__clz(m);  // starts are sorted: ok is a prefix
        lo = lo + last * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

// f(box, element index inside the box, segment) for every element of the
// span.  Chunks go to CTAs cyclically, so the CTAs running at any moment work
// on neighbouring chunks (the same few boxes, whose data then stays in L2).
// Each warp looks up the segment of its first element itself (no block
// barrier) and its lanes walk forward from there.
template <class F>
__device__ __forceinline__ void for_span(const Span& sp, F f) {
    const uint64_t chunk = (uint64_t)blockDim.x * kSpanItems;
    const uint64_t warp0 = threadIdx.x & ~31u;
    for (uint64_t g0 = (uint64_t)blockIdx.x * chunk; g0 < sp.total;
         g0 += (uint64_t)gridDim.x * chunk) {
        const uint64_t gw = g0 + warp0 < sp.total ? g0 + warp0 : g0;
        uint32_t k = seg_of_warp(sp, gw);
        for (int it = 0; it < kSpanItems; ++it) {
            const uint64_t g = g0 + (uint64_t)it * blockDim.x + threadIdx.x;
            if (g >= sp.total) break;
            while (g >= sp.start[k + 1]) ++k;
            f(sp.box[k], (uint64_t)sp.base[k] + (g - sp.start[k]), k);
        }
    }
}

static unsigned span_grid(const Span& sp) { return grid_for((sp.total + kSpanItems - 1) / kSpanItems); }

// One resident wave of span kernel K (grid_wave), never more than the span needs.
template <auto K>
static unsigned span_wave(const Span& sp) {
    return grid_wave<K>((sp.total + kSpanItems - 1) / kSpanItems);
}

#define SPAN_KERNEL(name, ...)                                                        \
    __global__ void __launch_bounds__(kBlock) name(Span sp, BatchArgs A) {            \
        for_span(sp, [&](uint32_t b, uint64_t i, uint32_t k) {                        \
            const BoxDev& D = A.dev[b];                                               \
            const BoxStep& S = A.step[b];                                             \
            (void)D;                                                                  \
            (void)S;                                                                  \
            (void)k;                                                                  \
            __VA_ARGS__                                                               \
        });                                                                           \
    }

#define SPAN_LAUNCH(fn, kern)                                        \
    void fn(cudaStream_t st, const Span& sp, const BatchArgs& a) {   \
        if (sp.total == 0) return;                                   \
        note_launch();                                               \
        kern<<<span_wave<kern>(sp), kBlock, 0, st>>>(sp, a);         \
    }

// ---- integrate --------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) kb_initial(Span sp, BatchArgs A) {
    for_span(sp, [&](uint32_t b, uint64_t i, uint32_t k) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const uint8_t f = sp.flag[k];
        const AtomCols& c = D.set[S.post];  // current at the start of a step
        double x, y, z;
        initial_atom(c, i, S.dt, (f & 2) != 0, (f & 4) != 0, x, y, z);
        if ((f & 1) && moved_too_far(x, y, z, D.lbx[i], D.lby[i], D.lbz[i], S.box, S.ibox, S.thr_sq))
            atomicOr(&A.flags[b].rebuild, 1u);
    });
}
SPAN_LAUNCH(b_initial, kb_initial)

SPAN_KERNEL(kb_final, { final_atom(D.set[S.post], i, S.dt); })
SPAN_LAUNCH(b_final, kb_final)

// soil_deform/src/lib.rs:568-574 (first shear step)
SPAN_KERNEL(kb_profile, {
    const AtomCols& c = D.set[S.post];
    c.vx[i] = c.vx[i] + D.shear_rate * (c.y[i] - D.yc);
})
SPAN_LAUNCH(b_profile, kb_profile)

SPAN_KERNEL(kb_zero_forces, {
    const AtomCols& c = D.set[S.cur];
    c.fx[i] = 0.0;
    c.fy[i] = 0.0;
    c.fz[i] = 0.0;
    for (int q = 0; q < D.zero.n; ++q) c.planes[D.zero.idx[q]][i] = 0.0;
})
SPAN_LAUNCH(b_zero_forces, kb_zero_forces)

SPAN_KERNEL(kb_pbc, { pbc_atom(D.set[S.cur], i, S.geom, S.bvel[0], S.bvel[1], S.bvel[2]); })
SPAN_LAUNCH(b_pbc, kb_pbc)

// ---- bins -----------------------------------------------------------------
__device__ __forceinline__ uint32_t* counts_of(const BoxDev& D, int which) {
    if (which == BA_IN) return D.in_count;
    return D.cell_counts;
}

__global__ void __launch_bounds__(kBlock) kb_zero_counts(Span sp, BatchArgs A, int which) {
    for_span(sp, [&](uint32_t b, uint64_t i, uint32_t) { counts_of(A.dev[b], which)[i] = 0u; });
}
void b_zero_counts(cudaStream_t st, const Span& sp, const BatchArgs& a, int which) {
    if (sp.total == 0) return;
    note_launch();
    kb_zero_counts<<<span_wave<kb_zero_counts>(sp), kBlock, 0, st>>>(sp, a, which);
}

__global__ void __launch_bounds__(kBlock) kb_cells(Span sp, BatchArgs A, int neighbor) {
    for_span(sp, [&](uint32_t b, uint64_t i, uint32_t) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const AtomCols& c = D.set[neighbor ? S.post : S.cur];
        const uint32_t cell = cell_of(S.grid, c.x[i], c.y[i], c.z[i]);
        (neighbor ? D.atom_cell : D.sort_cell)[i] = cell;
        atomicAdd(&D.cell_counts[cell], 1u);
    });
}
void b_cells(cudaStream_t st, const Span& sp, const BatchArgs& a, bool neighbor) {
    if (sp.total == 0) return;
    note_launch();
    kb_cells<<<span_wave<kb_cells>(sp), kBlock, 0, st>>>(sp, a, neighbor ? 1 : 0);
}

SPAN_KERNEL(kb_copy_count_local_cells, {
    const uint32_t cell = D.sorted_local_cell[i];
    D.atom_cell[i] = cell;
    atomicAdd(&D.cell_counts[cell], 1u);
})
SPAN_LAUNCH(b_copy_count_local_cells, kb_copy_count_local_cells)

// One CTA per segment: out = exclusive scan of in over the segment's n
// elements (out[n] = total), optional cursor copy.  Each thread takes
// kScanItems consecutive elements per pass (two 16-byte loads when the group
// is whole; every array is its own allocation, so element 0 is 256-byte
// aligned).  One CTA per segment lets the block scheduler balance boxes of
// very different sizes; spans list the largest boxes first.
constexpr int kScanItems = 8;

__global__ void __launch_bounds__(kBlock) kb_scan(Span sp, BatchArgs A, int which) {
    __shared__ uint32_t tot;
    const uint32_t k = blockIdx.x;
    const uint32_t b = sp.box[k];
    const BoxDev& D = A.dev[b];
    const uint64_t n = sp.start[k + 1] - sp.start[k];
    const uint32_t* in;
    uint32_t *out, *cursor;
    if (which == BA_ROWS) { in = D.rowcount; out = D.offsets; cursor = nullptr; }
    else if (which == BA_IN) { in = D.in_count; out = D.in_start; cursor = D.in_cursor; }
    else if (which == BA_GRP) { in = D.grp_cnt; out = D.grp_start; cursor = nullptr; }
    else { in = D.cell_counts; out = D.cell_start; cursor = D.cell_cursor; }
    uint32_t carry = 0;
    for (uint64_t b0 = 0; b0 < n; b0 += (uint64_t)kBlock * kScanItems) {
        const uint64_t t0 = b0 + (uint64_t)threadIdx.x * kScanItems;
        uint32_t v[kScanItems];
        const bool whole = t0 + kScanItems <= n;
        if (whole) {
            const uint4 p = *reinterpret_cast<const uint4*>(in + t0);
            const uint4 q = *reinterpret_cast<const uint4*>(in + t0 + 4);
            v[0] = p.x; v[1] = p.y; v[2] = p.z; v[3] = p.w;
            v[4] = q.x; v[5] = q.y; v[6] = q.z; v[7] = q.w;
        } else {
            for (int j = 0; j < kScanItems; ++j) v[j] = t0 + j < n ? in[t0 + j] : 0u;
        }
        uint32_t sum = 0;
        for (int j = 0; j < kScanItems; ++j) sum += v[j];
        uint32_t run = block_exclusive_scan(sum, &tot) + carry;
        for (int j = 0; j < kScanItems; ++j) {
            const uint32_t x = v[j];
            v[j] = run;
            run += x;
        }
        if (whole) {
            const uint4 p = make_uint4(v[0], v[1], v[2], v[3]);
            const uint4 q = make_uint4(v[4], v[5], v[6], v[7]);
            *reinterpret_cast<uint4*>(out + t0) = p;
            *reinterpret_cast<uint4*>(out + t0 + 4) = q;
            if (cursor) {
                *reinterpret_cast<uint4*>(cursor + t0) = p;
                *reinterpret_cast<uint4*>(cursor + t0 + 4) = q;
            }
        } else {
            for (int j = 0; j < kScanItems; ++j)
                if (t0 + j < n) {
                    out[t0 + j] = v[j];
                    if (cursor) cursor[t0 + j] = v[j];
                }
        }
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[n] = carry;
        if (which == BA_ROWS) A.totals[b] = carry;
    }
}
void b_scan(cudaStream_t st, const Span& sp, const BatchArgs& a, int which) {
    if (sp.nseg == 0) return;
    note_launch();
    kb_scan<<<sp.nseg, kBlock, 0, st>>>(sp, a, which);
}

__global__ void __launch_bounds__(kBlock) kb_scatter(Span sp, BatchArgs A, int neighbor) {
    for_span(sp, [&](uint32_t b, uint64_t i, uint32_t) {
        const BoxDev& D = A.dev[b];
        const uint32_t cell = (neighbor ? D.atom_cell : D.sort_cell)[i];
        (neighbor ? D.sorted_atoms : D.sort_perm)[atomicAdd(&D.cell_cursor[cell], 1u)] = (uint32_t)i;
    });
}
void b_scatter(cudaStream_t st, const Span& sp, const BatchArgs& a, bool neighbor) {
    if (sp.total == 0) return;
    note_launch();
    kb_scatter<<<span_wave<kb_scatter>(sp), kBlock, 0, st>>>(sp, a, neighbor ? 1 : 0);
}

__global__ void __launch_bounds__(kBlock) kb_segsort(Span sp, BatchArgs A, int which) {
    for_span(sp, [&](uint32_t b, uint64_t s, uint32_t) {
        const BoxDev& D = A.dev[b];
        if (which == BA_IN) insertion_sort(D.in_list, D.in_start[s], D.in_start[s + 1]);
        else insertion_sort(which == BA_NEIGH_CELLS ? D.sorted_atoms : D.sort_perm,
                            D.cell_start[s], D.cell_start[s + 1]);
    });
}
void b_segsort(cudaStream_t st, const Span& sp, const BatchArgs& a, int which) {
    if (sp.total == 0) return;
    note_launch();
    kb_segsort<<<span_wave<kb_segsort>(sp), kBlock, 0, st>>>(sp, a, which);
}

SPAN_KERNEL(kb_permute_cells, { D.sorted_local_cell[i] = D.sort_cell[D.sort_perm[i]]; })
SPAN_LAUNCH(b_permute_cells, kb_permute_cells)

SPAN_KERNEL(kb_identity, {
    if (D.sort_perm[i] != (uint32_t)i) atomicOr(&A.flags[b].not_identity, 1u);
})
SPAN_LAUNCH(b_identity, kb_identity)

SPAN_KERNEL(kb_perm_gather, { perm_gather_atom(D.set[S.cur], D.set[S.post], i, D.sort_perm[i]); })
SPAN_LAUNCH(b_perm_gather, kb_perm_gather)

// ---- borders (chain categories; the single-system kernels are in k_ghost.cu) ---
// Warp-tile spans: every warp takes one tile of 32 locals of one box;
// f(box, warp tile index inside the box, segment).
template <class F>
__device__ __forceinline__ void for_warp_tiles(const Span& sp, F f) {
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x / 32);
    for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; g < sp.total;
         g += nwarps) {
        const uint32_t k = seg_of_warp(sp, g);
        f(sp.box[k], (uint64_t)sp.base[k] + (g - sp.start[k]), k);
    }
}

__global__ void __launch_bounds__(kBlock) kb_border_faces(Span sp, BatchArgs A, BorderCats cats) {
    const uint32_t lane = threadIdx.x & 31u;
    for_warp_tiles(sp, [&](uint32_t b, uint64_t w, uint32_t k) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const uint64_t nw = sp.start[k + 1] - sp.start[k];
        border_warp_counts(D.set[S.post], S.nlocal, S.geom, S.geom.triclinic, S.thresh_lo,
                           S.thresh_hi, cats, D.face_flags, D.bcount, nw, w, lane);
    });
}
void b_border_faces(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.total == 0) return;
    note_launch();
    kb_border_faces<<<grid_wave<kb_border_faces>(sp.total * 32), kBlock, 0, st>>>(sp, a, border_cats());
}

// one CTA per (box, category): exclusive scan of the warp counts
__global__ void __launch_bounds__(kBlock) kb_border_cat_scan(Span sp, BatchArgs A) {
    const uint32_t seg = blockIdx.x / (kBorderCats + 1), k = blockIdx.x % (kBorderCats + 1);
    const uint32_t b = sp.box[seg];
    const BoxDev& D = A.dev[b];
    const uint64_t nw = sp.start[seg + 1] - sp.start[seg];
    const uint32_t total = cta_scan_array<8>(D.bcount + k * nw, D.boff + k * nw, nullptr, nw);
    if (threadIdx.x == 0) A.bstate[(uint64_t)b * kBorderStateWords + kBorderTotals + k] = total;
}
void b_border_cat_scan(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.nseg == 0) return;
    note_launch();
    kb_border_cat_scan<<<sp.nseg * (kBorderCats + 1), kBlock, 0, st>>>(sp, a);
}

__global__ void __launch_bounds__(kBlock) kb_border_images(Span sp, BatchArgs A, BorderCats cats) {
    __shared__ BorderWarpSmem sm[kBlock / 32];
    const uint32_t lane = threadIdx.x & 31u;
    for_warp_tiles(sp, [&](uint32_t b, uint64_t w, uint32_t k) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        uint32_t* bs = A.bstate + (uint64_t)b * kBorderStateWords;
        const uint64_t nw = sp.start[k + 1] - sp.start[k];
        if (w == 0 && lane == 0) border_state_words(cats, S.nlocal, bs);
        const uint32_t tot = lane < kBorderCats ? bs[kBorderTotals + lane] : 0u;
        const uint32_t base_lane = (uint32_t)S.nlocal + warp_exclusive_sum(tot, lane);
        border_warp_images(D.set[S.post], S.nlocal, D.cap, S.sc.off, S.sc.voff, cats, D.face_flags,
                           D.boff, nullptr, 1, nw, w, lane, base_lane, bs, D.ghost_root,
                           D.ghost_chain, D.send, D.fold_start, D.fold_list, sm[threadIdx.x / 32]);
    });
}
void b_border_images(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.total == 0) return;
    note_launch();
    kb_border_images<<<grid_wave<kb_border_images>(sp.total * 32), kBlock, 0, st>>>(sp, a, border_cats());
}

SPAN_KERNEL(kb_forward, {
    forward_ghost(D.set[S.post], S.nlocal, i, D.ghost_root, D.ghost_chain, S.sc, D.fwd, false);
})
SPAN_LAUNCH(b_forward, kb_forward)

// ---- neighbor build ---------------------------------------------------------
SPAN_KERNEL(kb_save_positions, {
    const AtomCols& c = D.set[S.post];
    D.lbx[i] = c.x[i];
    D.lby[i] = c.y[i];
    D.lbz[i] = c.z[i];
})
SPAN_LAUNCH(b_save_positions, kb_save_positions)

SPAN_KERNEL(kb_sorted_views, {
    sorted_view(D.set[S.post], i, D.sorted_atoms, D.asi, D.sp, S.filter ? D.spf : nullptr,
                S.geom.lo[0], S.geom.lo[1], S.geom.lo[2], BuildPos{}, S.uniform != 0);
})
SPAN_LAUNCH(b_sorted_views, kb_sorted_views)

__device__ __forceinline__ PairParams pair_params(const BoxDev& D, const BoxStep& S) {
    PairParams p;
    p.atom_cell = D.atom_cell;
    p.atom_sorted_idx = D.asi;
    p.bin_start = D.cell_start;
    p.sorted_atoms = D.sorted_atoms;
    p.sp = D.sp;
    p.spf = D.spf;
    p.stencil = S.stencil;
    p.nstencil = S.nstencil;
    p.ncells = S.ncells;
    p.nlocal = S.nlocal;
    p.has_self = S.has_self;
    p.newton = S.newton;
    p.uniform = S.uniform;
    p.filter = S.filter;
    p.row_slots = soil_host::kRowSlotsPerAtom;
    p.cut_sq = S.cut_sq;
    p.sf_sq = S.sf_sq;
    p.sf = S.sf;
    p.eps32 = S.eps32;
    p.in_count = nullptr;
    p.in_start = nullptr;
    p.in_list = nullptr;
    p.pre_ranges = S.pre_ranges;
    return p;
}

template <bool UNIFORM, bool FP32>
__device__ __forceinline__ void pairs_row(const PairParams& p, uint64_t i, uint32_t* rowcount,
                                          uint32_t* slots, DevFlags* flags, uint32_t& cd,
                                          uint32_t& rk) {
    const Filter<UNIFORM, FP32> test(p);
    const uint32_t K = (uint32_t)p.row_slots;
    rowcount[i] = row_scan<UNIFORM, FP32, true>(p, test, i, slots + i * K, K, &rk, &cd, flags);
}

__device__ __forceinline__ void add_filter_stats(DevFlags* f, uint32_t cd, uint32_t rk) {
    if (cd) atomicAdd((unsigned long long*)&f->candidates, (unsigned long long)cd);
    if (rk) atomicAdd((unsigned long long*)&f->rechecked, (unsigned long long)rk);
}

// Pair count pass over the rows of every box in the span.  The candidate and
// recheck statistics are summed per box inside each warp (lanes matched by
// box) before one atomic per box and warp.
__global__ void __launch_bounds__(kBlock) kb_pairs_rows(Span sp, BatchArgs A) {
    const uint64_t chunk = (uint64_t)blockDim.x * kSpanItems;
    const uint64_t warp0 = threadIdx.x & ~31u;
    for (uint64_t g0 = (uint64_t)blockIdx.x * chunk; g0 < sp.total;
         g0 += (uint64_t)gridDim.x * chunk) {
        const uint64_t gw = g0 + warp0 < sp.total ? g0 + warp0 : g0;
        uint32_t k = seg_of_warp(sp, gw);
        uint32_t cur = 0xffffffffu, cd = 0, rk = 0;
        for (int it = 0; it < kSpanItems; ++it) {
            const uint64_t g = g0 + (uint64_t)it * blockDim.x + threadIdx.x;
            if (g >= sp.total) break;
            while (g >= sp.start[k + 1]) ++k;
            const uint32_t b = sp.box[k];
            const uint64_t i = (uint64_t)sp.base[k] + (g - sp.start[k]);
            if (b != cur) {
                if (cur != 0xffffffffu) add_filter_stats(A.flags + cur, cd, rk);
                cur = b;
                cd = 0;
                rk = 0;
            }
            const BoxDev& D = A.dev[b];
            const BoxStep& S = A.step[b];
            const PairParams p = pair_params(D, S);
            DevFlags* fl = A.flags + b;
            if (S.uniform) {
                if (S.filter) pairs_row<true, true>(p, i, D.rowcount, D.row_slots, fl, cd, rk);
                else pairs_row<true, false>(p, i, D.rowcount, D.row_slots, fl, cd, rk);
            } else {
                if (S.filter) pairs_row<false, true>(p, i, D.rowcount, D.row_slots, fl, cd, rk);
                else pairs_row<false, false>(p, i, D.rowcount, D.row_slots, fl, cd, rk);
            }
        }
        const unsigned peers = __match_any_sync(0xffffffffu, cur);
        const uint32_t scd = __reduce_add_sync(peers, cd);
        const uint32_t srk = __reduce_add_sync(peers, rk);
        if (cur != 0xffffffffu && (int)(threadIdx.x & 31) == __ffs(peers) - 1)
            add_filter_stats(A.flags + cur, scd, srk);
    }
}
SPAN_LAUNCH(b_pairs_rows, kb_pairs_rows)

// The staged pair count over warp tiles of every box (the single-system
// kernel is k_pairs_staged); boxes whose stencil does not fit PairSegs scan
// their rows from global memory.
template <bool UNIFORM, bool FP32>
__device__ __forceinline__ bool batch_tile(const PairParams& p, const BoxStep& S, const BoxDev& D,
                                           uint64_t w, unsigned char* recs, uint64_t* bar,
                                           uint32_t& phase, uint32_t* lo, uint32_t* base,
                                           DevFlags* fl, uint32_t& cd, uint32_t& rk) {
    if (S.segs_ok)
        return staged_tile<UNIFORM, FP32>(p, S.segs, w, recs, bar, phase, lo, base, D.rowcount,
                                          D.row_slots, fl, rk, cd);
    const uint64_t i = w * 32 + (threadIdx.x & 31);
    if (i < p.nlocal) pairs_row<UNIFORM, FP32>(p, i, D.rowcount, D.row_slots, fl, cd, rk);
    return true;
}

__global__ void __launch_bounds__(kStageWarps * 32) kb_pairs_staged(Span sp, BatchArgs A) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint32_t s_lo[kStageWarps][kMaxPairSegs];
    __shared__ uint32_t s_base[kStageWarps][kMaxPairSegs];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char* recs = smem_raw + (size_t)wib * kStageRecs * 32;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + (size_t)kStageWarps * kStageRecs * 32) + wib;
    staged_init(bar);
    uint32_t phase = 0;
    bool ok = true;
    for_warp_tiles(sp, [&](uint32_t b, uint64_t w, uint32_t) {
        if (!ok) return;
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const PairParams p = pair_params(D, S);
        DevFlags* fl = A.flags + b;
        uint32_t cd = 0, rk = 0;
        if (S.uniform) {
            if (S.filter) ok = batch_tile<true, true>(p, S, D, w, recs, bar, phase, s_lo[wib], s_base[wib], fl, cd, rk);
            else ok = batch_tile<true, false>(p, S, D, w, recs, bar, phase, s_lo[wib], s_base[wib], fl, cd, rk);
        } else {
            if (S.filter) ok = batch_tile<false, true>(p, S, D, w, recs, bar, phase, s_lo[wib], s_base[wib], fl, cd, rk);
            else ok = batch_tile<false, false>(p, S, D, w, recs, bar, phase, s_lo[wib], s_base[wib], fl, cd, rk);
        }
        const uint32_t scd = __reduce_add_sync(0xffffffffu, cd);
        const uint32_t srk = __reduce_add_sync(0xffffffffu, rk);
        if (lane == 0) add_filter_stats(fl, scd, srk);
    });
}

void b_pairs_staged(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.total == 0) return;
    note_launch();
    const size_t smem = (size_t)kStageWarps * kStageRecs * 32 + kStageWarps * sizeof(uint64_t);
    const uint64_t per = kStageWarps;
    uint64_t blocks = (sp.total + per - 1) / per;
    if (blocks > 148ull * 8ull) blocks = 148ull * 8ull;
    kb_pairs_staged<<<(unsigned)blocks, kStageWarps * 32, smem, st>>>(sp, a);
}

template <bool UNIFORM, bool FP32>
__device__ __forceinline__ void fill_row(const PairParams& p, uint64_t i, const uint32_t* rowcount,
                                         const uint32_t* slots, const uint32_t* offsets,
                                         uint32_t* indices) {
    const uint32_t K = (uint32_t)p.row_slots;
    const uint32_t cnt = rowcount[i];
    uint32_t* out = indices + offsets[i];
    if (cnt <= K) {
        const uint32_t* row = slots + i * K;
        for (uint32_t q = 0; q < cnt; ++q) out[q] = row[q];
    } else {
        const Filter<UNIFORM, FP32> test(p);
        uint32_t rk = 0, cd = 0;
        row_scan<UNIFORM, FP32, true>(p, test, i, out, 0xffffffffu, &rk, &cd, nullptr);
    }
}

SPAN_KERNEL(kb_pairs_fill, {
    const PairParams p = pair_params(D, S);
    if (S.uniform) {
        if (S.filter) fill_row<true, true>(p, i, D.rowcount, D.row_slots, D.offsets, D.indices);
        else fill_row<true, false>(p, i, D.rowcount, D.row_slots, D.offsets, D.indices);
    } else {
        if (S.filter) fill_row<false, true>(p, i, D.rowcount, D.row_slots, D.offsets, D.indices);
        else fill_row<false, false>(p, i, D.rowcount, D.row_slots, D.offsets, D.indices);
    }
})
SPAN_LAUNCH(b_pairs_fill, kb_pairs_fill)

SPAN_KERNEL(kb_in_count, {
    for (uint32_t q = D.offsets[i]; q < D.offsets[i + 1]; ++q) atomicAdd(&D.in_count[D.indices[q]], 1u);
})
SPAN_LAUNCH(b_in_count, kb_in_count)

SPAN_KERNEL(kb_in_scatter, {
    for (uint32_t q = D.offsets[i]; q < D.offsets[i + 1]; ++q)
        D.in_list[atomicAdd(&D.in_cursor[D.indices[q]], 1u)] = (uint32_t)i;
})
SPAN_LAUNCH(b_in_scatter, kb_in_scatter)

// ---- force and reverse comm ---------------------------------------------------
// Register-capped like the single-system force kernel (5 blocks per SM) and
// launched as one resident wave.
__global__ void __launch_bounds__(kBlock, 5) kb_harmonic(Span sp, BatchArgs A) {
    for_span(sp, [&](uint32_t b, uint64_t i, uint32_t) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const AtomCols& c = D.set[S.post];
        harmonic_atom(c, i, S.nlocal, c.planes[D.radius_plane], S.K, S.newton, D.offsets,
                      D.indices, D.in_start, D.in_list);
    });
}
void b_harmonic(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.total == 0) return;
    note_launch();
    const unsigned g = span_grid(sp);
    kb_harmonic<<<g < 148u * 5u ? g : 148u * 5u, kBlock, 0, st>>>(sp, a);
}

SPAN_KERNEL(kb_reverse, { fold_root(D.set[S.post], S.nlocal, i, D.fold_start, D.fold_list, D.rev); })
SPAN_LAUNCH(b_reverse, kb_reverse)

// ---- the grouped consumer (the single-system kernels are in k_force.cu) -------
__device__ __forceinline__ SeqArgs seq_args(const BoxDev& D, const BoxStep& S) {
    SeqArgs q;
    q.nlocal = S.nlocal;
    q.ntotal = S.nlocal + S.nghost;
    q.newton = S.newton;
    q.offsets = D.offsets;
    q.indices = D.indices;
    q.in_start = D.in_start;
    q.in_list = D.in_list;
    q.fold_start = D.fold_start;
    q.fold_list = D.fold_list;
    return q;
}

SPAN_KERNEL(kb_seq_count, { seq_count_atom(seq_args(D, S), i, D.seq_cnt, D.grp_cnt); })
SPAN_LAUNCH(b_seq_count, kb_seq_count)

SPAN_KERNEL(kb_seq_fill, { seq_fill_root(seq_args(D, S), i, D.grp_start, D.seq, D.seq_owner); })
SPAN_LAUNCH(b_seq_fill, kb_seq_fill)

__device__ __forceinline__ ForceSeq force_seq_of(const BoxDev& D, const BoxStep& S,
                                                 const AtomCols& c) {
    ForceSeq q;
    q.rad = c.planes[D.radius_plane];
    q.K = S.K;
    q.nlocal = S.nlocal;
    q.grp_start = D.grp_start;
    q.cnt = D.seq_cnt;
    q.seq = D.seq;
    q.owner = D.seq_owner;
    q.fold_start = D.fold_start;
    q.fold_list = D.fold_list;
    q.pk = nullptr;
    return q;
}

__global__ void __launch_bounds__(kBlock, 3) kb_force_grouped(Span sp, BatchArgs A) {
    __shared__ ForceSmem<4> sm;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for_warp_tiles(sp, [&](uint32_t b, uint64_t w, uint32_t) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const AtomCols& c = D.set[S.post];
        const ForceSeq q = force_seq_of(D, S, c);
        if (S.newton) force_tile<4, true>(q, c, D.rev, w, sm, lane, wib);
        else force_tile<4, false>(q, c, D.rev, w, sm, lane, wib);
    });
}
__global__ void __launch_bounds__(kBlock, 4) kb_force_walk(Span sp, BatchArgs A) {
    for_span(sp, [&](uint32_t b, uint64_t i, uint32_t) {
        const BoxDev& D = A.dev[b];
        const BoxStep& S = A.step[b];
        const AtomCols& c = D.set[S.post];
        const ForceSeq q = force_seq_of(D, S, c);
        if (S.newton) force_walk_root<true, false>(q, c, D.rev, i);
        else force_walk_root<false, false>(q, c, D.rev, i);
    });
}
void b_force_walk(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.total == 0) return;
    note_launch();
    const unsigned g = span_grid(sp);
    kb_force_walk<<<g < 148u * 4u ? g : 148u * 4u, kBlock, 0, st>>>(sp, a);
}

void b_force_grouped(cudaStream_t st, const Span& sp, const BatchArgs& a) {
    if (sp.total == 0) return;
    note_launch();
    uint64_t blocks = (sp.total + kBlock / 32 - 1) / (kBlock / 32);
    if (blocks > 148ull * 3ull) blocks = 148ull * 3ull;  // one resident wave
    kb_force_grouped<<<(unsigned)blocks, kBlock, 0, st>>>(sp, a);
}

}  // namespace soil
