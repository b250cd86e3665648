// soil_capi.cu — host side of the soil_b200 library: the C ABI of
// include/soil_cuda.h, device memory of one system, and the timestep
// orchestration in the reference schedule order (schedule.rs:22-52):
//
//   PreInitialIntegration  apply_deform            soil_phase_deform
//   InitialIntegration     initial_integration     soil_phase_initial
//   PostInitialIntegration decide_rebuild, remove_ghost_atoms, zero_all_forces
//   PreExchange            pbc
//   PreNeighbor            sort_atoms_by_bin, borders | forward_comm_borders
//   Neighbor               bin_neighbor_list
//   Force                  force hook / built-in consumer
//   PostForce              reverse_send_force
//   FinalIntegration       final_integration
//
// Scalar bookkeeping (CommState, counters, bin grid, stencil, swap ranges)
// lives on the host exactly as in the reference resources; all per-atom work
// runs on the device.  The host reads back a few words where the reference
// branches on data: the displacement flag, the identity flag of a periodic
// sort, ghost totals and the pair total of a rebuild.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "sys_internal.cuh"

using namespace soil;

namespace soil_host {

int fail(soil_ctx* ctx, int status, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->err = buf;
    }
    return status;
}

// Reserve `bytes` of the context's HBM budget (thread-safe: the batch engine
// plans boxes on several host threads).
int ctx_reserve(soil_ctx* ctx, uint64_t bytes) {
    std::lock_guard<std::mutex> g(ctx->mu);
    if (ctx->budget && ctx->in_use + bytes > ctx->budget) {
        char buf[160];
        snprintf(buf, sizeof buf, "HBM budget exceeded: %llu + %llu > %llu bytes",
                 (unsigned long long)ctx->in_use, (unsigned long long)bytes,
                 (unsigned long long)ctx->budget);
        ctx->err = buf;
        return SOIL_ERR_OOM;
    }
    ctx->in_use += bytes;
    ctx->allocs += 1;
    return SOIL_OK;
}

void ctx_release(soil_ctx* ctx, uint64_t bytes) {
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->in_use -= bytes;
    ctx->frees += 1;
}

int dev_alloc(soil_sys* s, void** p, uint64_t bytes) {
    if (bytes == 0) bytes = 16;
    TRY(ctx_reserve(s->ctx, bytes));
    // stream-ordered from the context's pool: no device-wide synchronisation,
    // and freed memory stays in the pool for the next growth
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, s->ctx->pool, s->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx_release(s->ctx, bytes);
        return fail(s->ctx, SOIL_ERR_OOM, "cudaMallocAsync(%llu): %s", (unsigned long long)bytes,
                    cudaGetErrorString(e));
    }
    return SOIL_OK;
}

// Frees in stream order after every use already enqueued on the system's stream.
void dev_free(soil_sys* s, void* p, uint64_t bytes) {
    if (!p) return;
    cudaFreeAsync(p, s->st);
    if (bytes == 0) bytes = 16;
    ctx_release(s->ctx, bytes);
}

// ---- per-atom columns -------------------------------------------------------
constexpr int kDoubleCols = 12;  // x y z vx vy vz fx fy fz mass inv_mass cut
constexpr int kRowSlots = kRowSlotsPerAtom;  // neighbor entries per atom kept by the first pair pass

double** dcol(AtomCols& c, int k) {
    double** t[kDoubleCols] = {&c.x, &c.y, &c.z, &c.vx, &c.vy, &c.vz,
                               &c.fx, &c.fy, &c.fz, &c.mass, &c.inv_mass, &c.cut};
    return t[k];
}

void free_cols(soil_sys* s, AtomCols& c) {
    for (int k = 0; k < kDoubleCols; ++k) {
        dev_free(s, *dcol(c, k), c.cap * 8);
        *dcol(c, k) = nullptr;
    }
    dev_free(s, c.tag, c.cap * 4);
    dev_free(s, c.type, c.cap * 4);
    dev_free(s, c.img, c.cap * 12);
    dev_free(s, c.origin, c.cap * 4);
    // one block per registered column holds its planes
    for (const ColMeta& m : s->cols)
        if (m.plane0 < c.nplanes) dev_free(s, c.planes[m.plane0], c.cap * 8 * (uint64_t)m.width);
    for (int q = 0; q < c.nplanes; ++q) c.planes[q] = nullptr;
    c.tag = c.type = nullptr;
    c.img = c.origin = nullptr;
}

// Allocate a column set of capacity `cap`, copying [0, keep) from `old`.
// On failure nothing stays allocated.
int alloc_cols(soil_sys* s, AtomCols& c, uint64_t cap, const AtomCols* old, uint64_t keep) {
    AtomCols n{};
    n.cap = cap;
    n.nplanes = s->nplanes;
    int st = SOIL_OK;
    for (int k = 0; k < kDoubleCols && st == SOIL_OK; ++k) st = dev_alloc(s, (void**)dcol(n, k), cap * 8);
    if (st == SOIL_OK) st = dev_alloc(s, (void**)&n.tag, cap * 4);
    if (st == SOIL_OK) st = dev_alloc(s, (void**)&n.type, cap * 4);
    if (st == SOIL_OK) st = dev_alloc(s, (void**)&n.img, cap * 12);
    if (st == SOIL_OK) st = dev_alloc(s, (void**)&n.origin, cap * 4);
    // The planes of a column of width w are one block of w * cap doubles:
    // component k of atom i is planes[plane0][k * cap + i], the layout the
    // device view documents (columns[c][k * stride + i]).
    for (const ColMeta& m : s->cols) {
        if (st != SOIL_OK) break;
        double* blk = nullptr;
        st = dev_alloc(s, (void**)&blk, cap * 8 * (uint64_t)m.width);
        if (st == SOIL_OK)
            for (int k = 0; k < m.width; ++k) n.planes[m.plane0 + k] = blk + k * cap;
    }
    if (st != SOIL_OK) {
        free_cols(s, n);
        return st;
    }
    if (old && keep) {
        AtomCols o = *old;
        for (int k = 0; k < kDoubleCols; ++k)
            CK(cudaMemcpyAsync(*dcol(n, k), *dcol(o, k), keep * 8, cudaMemcpyDeviceToDevice, s->st));
        CK(cudaMemcpyAsync(n.tag, o.tag, keep * 4, cudaMemcpyDeviceToDevice, s->st));
        CK(cudaMemcpyAsync(n.type, o.type, keep * 4, cudaMemcpyDeviceToDevice, s->st));
        for (int d = 0; d < 3; ++d)
            CK(cudaMemcpyAsync(n.img + d * cap, o.img + d * o.cap, keep * 4, cudaMemcpyDeviceToDevice,
                               s->st));
        CK(cudaMemcpyAsync(n.origin, o.origin, keep * 4, cudaMemcpyDeviceToDevice, s->st));
        for (int q = 0; q < s->nplanes; ++q)
            CK(cudaMemcpyAsync(n.planes[q], o.planes[q], keep * 8, cudaMemcpyDeviceToDevice, s->st));
    }
    c = n;
    return SOIL_OK;
}

int update_colptrs(soil_sys* s) {
    if (s->cols.empty() || !s->colptrs_dirty) return SOIL_OK;
    TRY(ensure(s, s->d_colptrs, kMaxCols));
    double* h[kMaxCols] = {};
    for (size_t c = 0; c < s->cols.size(); ++c) h[c] = s->A.planes[s->cols[c].plane0];
    CK(cudaMemcpyAsync(s->d_colptrs.p, h, sizeof(h), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->colptrs_dirty = false;
    return SOIL_OK;
}

// Scratch of the ordered selections (atom removal, send lists of swaps with
// no neighbor, the reverse-comm root list), sized with the atom capacity.
int select_arrays(soil_sys* s) {
    TRY(ensure(s, s->sel_flag, s->acap + 1));
    TRY(ensure(s, s->sel_pos, s->acap + 2));
    TRY(ensure(s, s->sel_out, s->acap + 1));
    TRY(ensure(s, s->sel_cnt, kNumSwaps + 1));
    TRY(ensure(s, s->scan_tmp, scan_temp_words(s->acap + 2)));
    return SOIL_OK;
}

// Capacity for `need` atoms (locals + ghosts); the first `keep` survive.
int grow_atoms(soil_sys* s, uint64_t need, uint64_t keep) {
    if (need <= s->acap && s->A.x) return SOIL_OK;
    if (need >= 0x7fffffffull)
        return fail(s->ctx, SOIL_ERR_CAPACITY, "atom count %llu exceeds the u32 index range",
                    (unsigned long long)need);
    uint64_t ncap = need + need / 4 + 1024;
    AtomCols nA{}, nB{};
    TRY(alloc_cols(s, nA, ncap, s->A.x ? &s->A : nullptr, keep));
    const int st = alloc_cols(s, nB, ncap, nullptr, 0);
    if (st != SOIL_OK) {  // capacity unchanged: the new A goes back
        free_cols(s, nA);
        return st;
    }
    if (s->A.x) free_cols(s, s->A);  // after the copies above, in stream order
    if (s->B.x) free_cols(s, s->B);
    s->A = nA;
    s->B = nB;
    s->acap = ncap;
    // ghost-indexed arrays keep their [0, keep - nlocal) prefix
    uint64_t gkeep = keep > s->nlocal ? keep - s->nlocal : 0;
    TRY(ensure(s, s->ghost_root, ncap, gkeep));
    TRY(ensure(s, s->ghost_chain, ncap, gkeep));
    // The spatial sort's per-atom arrays follow the capacity, so a system's
    // first sort (often its first rebuild inside a run) allocates nothing.
    // Growth happens between a sort and the neighbor build that reuses its
    // local cells, so the locals' entries survive it.
    TRY(ensure(s, s->sort_cell, ncap, s->sort_cell.p ? std::min(keep, s->sort_cell.cap) : 0));
    TRY(ensure(s, s->sort_perm, ncap, s->sort_perm.p ? std::min(keep, s->sort_perm.cap) : 0));
    TRY(ensure(s, s->sorted_local_cell, ncap,
               s->sorted_local_cell.p ? std::min(keep, s->sorted_local_cell.cap) : 0));
    TRY(slots_grow(s, ncap, keep));
    // ordered-selection scratch and the reverse-comm root list, so that no
    // later phase allocates
    TRY(select_arrays(s));
    TRY(ensure(s, s->fold_roots, ncap + 1));
    TRY(ensure(s, s->fold_nroots, 1));
    s->colptrs_dirty = true;
    return SOIL_OK;
}

// Slot sets for `cap` atoms: the current set keeps its first `keep` rows and
// every later row is empty; the other set is scratch for the next writer.
int slots_grow(soil_sys* s, uint64_t cap, uint64_t keep) {
    if (!s->slot_max) return SOIL_OK;
    const uint64_t M = s->slot_max, W = s->slot_width;
    const int o = s->slot_old;
    if (!s->slot_tag[o].p) keep = 0;
    TRY(ensure(s, s->slot_tag[o], cap * M, keep * M));
    TRY(ensure(s, s->slot_val[o], cap * M * W, keep * M * W));
    TRY(ensure(s, s->slot_tag[1 - o], cap * M));
    TRY(ensure(s, s->slot_val[1 - o], cap * M * W));
    if (cap > keep) {
        CK(cudaMemsetAsync(s->slot_tag[o].p + keep * M, 0xFF, (cap - keep) * M * 4, s->st));
        CK(cudaMemsetAsync(s->slot_val[o].p + keep * M * W, 0, (cap - keep) * M * W * 8, s->st));
    }
    return SOIL_OK;
}

// ---- phase timers -------------------------------------------------------------
enum { T_INTEGRATE, T_ZERO, T_PBC, T_SORT, T_BORDERS, T_FORWARD, T_NEIGHBOR, T_FORCE, T_REVERSE,
       T_FINAL };
const char* kTimerNames[SOIL_NUM_TIMERS] = {"integrate", "zero",     "pbc",   "sort",    "borders",
                                            "forward",   "neighbor", "force", "reverse", "final"};

cudaEvent_t take_event(soil_sys* s) {
    if (s->ev_pool.empty()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return e;
    }
    cudaEvent_t e = s->ev_pool.back();
    s->ev_pool.pop_back();
    return e;
}

void timer_begin(soil_sys* s, int t) {
    if (!(s->timing_mask & (1u << t))) return;
    cudaEvent_t e = take_event(s);
    if (!e) return;
    cudaEventRecord(e, s->st);
    s->open_timer = t;
    s->open_ev = e;
    s->open_launches = launches_so_far();
}

void timer_end(soil_sys* s, int t) {
    if (s->open_timer != t) return;
    cudaEvent_t e = take_event(s);
    if (e) {
        cudaEventRecord(e, s->st);
        s->spans.push_back({t, s->open_ev, e, launches_so_far() - s->open_launches});
    } else {
        s->ev_pool.push_back(s->open_ev);
    }
    s->open_timer = -1;
}

// Fold completed spans into the sums (the stream must be idle).
void resolve_timers(soil_sys* s) {
    for (auto& sp : s->spans) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) {
            s->timer_ms[sp.timer] += ms;
            s->timer_launches[sp.timer] += sp.launches;
            s->timer_intervals[sp.timer] += 1;
        } else {
            cudaGetLastError();
        }
        s->ev_pool.push_back(sp.a);
        s->ev_pool.push_back(sp.b);
    }
    s->spans.clear();
}

int sync(soil_sys* s) {
    CK(cudaStreamSynchronize(s->st));
    CK(cudaGetLastError());
    return SOIL_OK;
}

// Largest count the single-pass scan takes (SOIL_SCAN1P_MAX overrides, for
// A/B runs; read at each call).
uint64_t scan1p_max() {
    const char* env = std::getenv("SOIL_SCAN1P_MAX");
    return env ? std::strtoull(env, nullptr, 10) : kScan1pMaxCounts;
}

int scan_1p(soil_sys* s, const uint32_t* in, uint32_t* out, uint64_t n) {
    // Up to 64 tiles of 2,048 counts the single launch saves launch latency;
    // above it the three-kernel scan is faster (the look-back of a thousand
    // resident CTAs contends).
    if (n > scan1p_max()) {
        TRY(ensure(s, s->scan_tmp, scan_temp_words(n + 2)));
        exclusive_scan_u32(s->st, in, out, n, s->scan_tmp.p);
        return SOIL_OK;
    }
    const uint64_t need = scan1p_words(n);
    if (!s->scan1p.p || s->scan1p.cap < need) {
        TRY(ensure(s, s->scan1p, need, 0, scan1p_words(2 * n + 4096)));
        CK(cudaMemsetAsync(s->scan1p.p, 0, s->scan1p.cap * 4, s->st));
    }
    exclusive_scan_1p(s->st, in, out, n, s->scan1p.p, &s->dflags->fault);
    return SOIL_OK;
}

// Two independent scans; above the single-pass size both go in the same two
// launches.
int scan_pair(soil_sys* s, const uint32_t* in0, uint32_t* out0, uint64_t n0, const uint32_t* in1,
              uint32_t* out1, uint64_t n1) {
    const uint64_t lim = scan1p_max();
    if (n0 > lim && n1 > lim) {
        TRY(ensure(s, s->scan_tmp, scan_temp_words(n0 + 2) + scan_temp_words(n1 + 2)));
        exclusive_scan_u32_pair(s->st, in0, out0, n0, in1, out1, n1, s->scan_tmp.p);
        return SOIL_OK;
    }
    TRY(scan_1p(s, in0, out0, n0));
    return scan_1p(s, in1, out1, n1);
}

int pairs_pre_ranges() {
    const char* env = std::getenv("SOIL_PAIRS_PRE");
    return env && std::atoi(env) == 0 ? 0 : 1;
}

std::vector<int32_t> stencil_runs(const std::vector<int32_t>& sten, bool newton) {
    std::vector<int32_t> r;
    for (const int32_t off : sten) {
        if (!newton && off == 0) continue;
        if (!r.empty() && r[r.size() - 2] + r.back() == off) {
            r.back() += 1;
            continue;
        }
        r.push_back(off);
        r.push_back(1);
    }
    return r;
}

int counts_zero(soil_sys* s, uint64_t nc) {
    if (s->counts_at != s->cell_counts.p || s->counts_clean < nc)
        CK(cudaMemsetAsync(s->cell_counts.p, 0, s->cell_counts.cap * 4, s->st));
    s->counts_at = s->cell_counts.p;
    s->counts_clean = 0;  // counted into now; clean again once consumed
    return SOIL_OK;
}

// After a consuming scatter over every counted atom: all counts are zero.
void counts_consumed(soil_sys* s) { s->counts_clean = s->cell_counts.cap; }

int check_launch(soil_sys* s) {
    CK(cudaGetLastError());
    return SOIL_OK;
}

Geom geom_of(const soil_sys* s) {
    Geom g;
    for (int d = 0; d < 3; ++d) {
        g.lo[d] = s->blo[d];
        g.size[d] = s->size[d];
        g.tilt[d] = s->tilt[d];
    }
    g.triclinic = s->triclinic ? 1 : 0;
    return g;
}

Grid grid_of(const soil_sys* s) {
    Grid gr;
    for (int d = 0; d < 3; ++d) {
        gr.origin[d] = s->bin_origin[d];
        gr.inv_bs[d] = 1.0 / s->bin_size[d];
        gr.n[d] = s->bin_count[d];
    }
    gr.geom = geom_of(s);
    return gr;
}

// ---- bin grid (host) ----------------------------------------------------------
// compute_bin_grid, neighbor.rs:311-397 (one rank)
void compute_bin_grid(soil_sys* s);

void compute_bin_grid_triclinic(soil_sys* s, double max_cutoff, double min_bin) {
    // neighbor.rs:411-495
    const double* l = s->size;
    const double xy = s->tilt[0];
    double sub_l[3];
    for (int d = 0; d < 3; ++d) sub_l[d] = s->sub_lam_hi[d] - s->sub_lam_lo[d];
    int32_t ni[3];
    for (int d = 0; d < 3; ++d) ni[d] = sat_i32(std::fmax(std::floor(sub_l[d] * l[d] / min_bin), 1.0));
    double bl[3], real_bin[3];
    for (int d = 0; d < 3; ++d) bl[d] = sub_l[d] / (double)ni[d];
    for (int d = 0; d < 3; ++d) real_bin[d] = bl[d] * l[d];
    const double ghost_cut = s->domain_ghost_cutoff > max_cutoff ? s->domain_ghost_cutoff : max_cutoff;
    int32_t sr[3];
    for (int d = 0; d < 3; ++d) sr[d] = sat_i32(std::ceil(max_cutoff / real_bin[d]));
    const int32_t skew = sat_i32(std::ceil(std::fabs(xy) / real_bin[0]));
    const int32_t sx = sat_i32(std::ceil(ghost_cut / real_bin[0])) + sr[0] + skew;
    const int32_t sy = sat_i32(std::ceil(ghost_cut / real_bin[1])) + sr[1];
    const int32_t sz = sat_i32(std::ceil(ghost_cut / real_bin[2])) + sr[2];
    const int32_t nx = ni[0] + 2 * sx, ny = ni[1] + 2 * sy, nz = ni[2] + 2 * sz;
    s->bin_count[0] = nx;
    s->bin_count[1] = ny;
    s->bin_count[2] = nz;
    for (int d = 0; d < 3; ++d) s->bin_size[d] = bl[d];
    s->total_cells = (uint64_t)(nx * ny * nz);
    s->bin_origin[0] = s->sub_lam_lo[0] - bl[0] * (double)sx;
    s->bin_origin[1] = s->sub_lam_lo[1] - bl[1] * (double)sy;
    s->bin_origin[2] = s->sub_lam_lo[2] - bl[2] * (double)sz;
    const double cutoff_sq = max_cutoff * max_cutoff;
    s->stencil.clear();
    s->stencil_fwd.clear();
    s->stencil_self = false;
    for (int32_t dx = -sx; dx <= sx; ++dx)
        for (int32_t dy = -sy; dy <= sy; ++dy)
            for (int32_t dz = -sz; dz <= sz; ++dz) {
                const double m1 = (double)(std::abs(dy) > 0 ? std::abs(dy) - 1 : 0) * bl[1];
                const double m2 = (double)(std::abs(dz) > 0 ? std::abs(dz) - 1 : 0) * bl[2];
                const double dyz_sq = (l[1] * m1) * (l[1] * m1) + (l[2] * m2) * (l[2] * m2);
                if (dyz_sq >= cutoff_sq) continue;
                const double budget = std::sqrt(cutoff_sq - dyz_sq);
                const double a_lo = l[0] * ((double)dx - 1.0) * bl[0];
                const double a_hi = l[0] * ((double)dx + 1.0) * bl[0];
                const double b1 = xy * ((double)dy - 1.0) * bl[1];
                const double b2 = xy * ((double)dy + 1.0) * bl[1];
                const double b_lo = b1 <= b2 ? b1 : b2;
                const double b_hi = b1 <= b2 ? b2 : b1;
                const double lo = a_lo + b_lo;
                const double hi = a_hi + b_hi;
                if (hi >= -budget && lo <= budget) {
                    const int32_t off = dx * ny * nz + dy * nz + dz;
                    s->stencil.push_back(off);
                    if (off > 0) s->stencil_fwd.push_back(off);
                    else if (off == 0) s->stencil_self = true;
                }
            }
    for (int d = 0; d < 3; ++d) s->pbc_box[d] = l[d];
}

void compute_bin_grid(soil_sys* s) {
    const double max_cutoff = s->cached_max_cutoff;
    const double min_bin = std::fmax(s->bin_min_size, max_cutoff);
    if (s->triclinic) {
        compute_bin_grid_triclinic(s, max_cutoff, min_bin);
        return;
    }
    int32_t ni[3];
    double abs_[3];
    for (int d = 0; d < 3; ++d) ni[d] = sat_i32(std::fmax(std::floor(s->sub_len[d] / min_bin), 1.0));
    for (int d = 0; d < 3; ++d) abs_[d] = s->sub_len[d] / (double)ni[d];
    const double ghost_cut = s->domain_ghost_cutoff > max_cutoff ? s->domain_ghost_cutoff : max_cutoff;
    int32_t sv[3];
    for (int d = 0; d < 3; ++d)
        sv[d] = sat_i32(std::ceil(ghost_cut / abs_[d])) + sat_i32(std::ceil(max_cutoff / abs_[d]));
    const int32_t nx = ni[0] + 2 * sv[0], ny = ni[1] + 2 * sv[1], nz = ni[2] + 2 * sv[2];
    s->bin_count[0] = nx;
    s->bin_count[1] = ny;
    s->bin_count[2] = nz;
    for (int d = 0; d < 3; ++d) s->bin_size[d] = abs_[d];
    s->total_cells = (uint64_t)(nx * ny * nz);
    for (int d = 0; d < 3; ++d) s->bin_origin[d] = s->sub_lo[d] - abs_[d] * (double)sv[d];
    const double cutoff_sq = max_cutoff * max_cutoff;
    s->stencil.clear();
    s->stencil_fwd.clear();
    s->stencil_self = false;
    for (int32_t dx = -sv[0]; dx <= sv[0]; ++dx)
        for (int32_t dy = -sv[1]; dy <= sv[1]; ++dy)
            for (int32_t dz = -sv[2]; dz <= sv[2]; ++dz) {
                const double mdx = (double)(std::abs(dx) > 0 ? std::abs(dx) - 1 : 0) * abs_[0];
                const double mdy = (double)(std::abs(dy) > 0 ? std::abs(dy) - 1 : 0) * abs_[1];
                const double mdz = (double)(std::abs(dz) > 0 ? std::abs(dz) - 1 : 0) * abs_[2];
                if (mdx * mdx + mdy * mdy + mdz * mdz < cutoff_sq) {
                    const int32_t off = dx * ny * nz + dy * nz + dz;
                    s->stencil.push_back(off);
                    if (off > 0) s->stencil_fwd.push_back(off);
                    else if (off == 0) s->stencil_self = true;
                }
            }
    for (int d = 0; d < 3; ++d) s->pbc_box[d] = s->bhi[d] - s->blo[d];
}

double displacement_threshold_sq(const soil_sys* s) {
    // displacement_exceeded, neighbor.rs:700-702; additive_skin adds s/2 per atom
    double per_atom_skin = (s->skin_fraction - 1.0) * s->cached_min_skin;
    if (s->additive_skin != 0.0) per_atom_skin = per_atom_skin + 0.5 * s->additive_skin;
    return per_atom_skin * per_atom_skin;
}

void zero_planes_of(const soil_sys* s, unsigned flag, int* out, int* n) {
    *n = 0;
    for (const ColMeta& c : s->cols)
        if (c.flags & flag)
            for (int w = 0; w < c.width; ++w) out[(*n)++] = c.plane0 + w;
}

bool builtin_consumer(const soil_sys* s) {
    return s->hook == nullptr && s->harmonic_k != 0.0 && s->radius_col >= 0;
}

// ---------------------------------------------------------------------------
// Phases
// ---------------------------------------------------------------------------
// apply_deform xy branch, soil_deform/src/lib.rs:435-604, host part.  Returns
// true when the one-time streaming profile must be applied to the locals.
bool has_axis_deform(const soil_sys* s) {
    return s->axis[0].style || s->axis[1].style || s->axis[2].style;
}

// apply_deform (soil_deform/src/lib.rs:435-604) on the host state: the
// orthogonal axes (lib.rs:468-557; the position remap is returned in r for
// the device), then the xy shear.  *profile: the one-time streaming profile
// is due this step.
int deform_step(soil_sys* s, bool* profile, RemapSpec* r) {
    *profile = false;
    r->n = 0;
    if (!s->deform_initialized || !(s->shear || has_axis_deform(s))) return SOIL_OK;
    s->deform_step += 1;
    const uint64_t step = s->deform_step;
    bool box_changed = false;
    for (int dim = 0; dim < 3; ++dim) {
        const soil_sys::AxisDeform& ax = s->axis[dim];
        if (!ax.style) continue;
        const double old_lo = s->blo[dim], old_hi = s->bhi[dim];
        const double old_size = old_hi - old_lo;
        const double l0 = ax.hi0 - ax.lo0;
        double new_lo, new_hi;
        if (ax.style == SOIL_DEFORM_ERATE) {
            const double scale = 1.0 + ax.a * s->dt * (double)step;
            const double new_l = l0 * scale;
            const double center = (ax.lo0 + ax.hi0) * 0.5;
            new_lo = center - new_l * 0.5;
            new_hi = center + new_l * 0.5;
        } else if (ax.style == SOIL_DEFORM_VEL) {
            const double delta = ax.a * s->dt * (double)step;
            const double new_l = l0 + delta;
            const double center = (ax.lo0 + ax.hi0) * 0.5;
            new_lo = center - new_l * 0.5;
            new_hi = center + new_l * 0.5;
        } else {
            double frac = ax.stage_steps > 0 ? (double)step / (double)ax.stage_steps : 1.0;
            frac = std::fmin(frac, 1.0);
            new_lo = ax.lo0 + (ax.a - ax.lo0) * frac;
            new_hi = ax.hi0 + (ax.b - ax.hi0) * frac;
        }
        const double new_size = new_hi - new_lo;
        if (new_size <= 0.0)
            return fail(s->ctx, SOIL_ERR_INVALID, "deform: axis %c collapsed at step %llu",
                        "xyz"[dim], (unsigned long long)step);
        if (s->remap && old_size > 0.0) {
            const int q = r->n++;
            r->dim[q] = dim;
            r->scale[q] = new_size / old_size;
            r->new_center[q] = (new_lo + new_hi) * 0.5;
            r->old_center[q] = (old_lo + old_hi) * 0.5;
        }
        s->blo[dim] = new_lo;
        s->bhi[dim] = new_hi;
        s->size[dim] = new_size;
        s->sub_lo[dim] = new_lo;
        s->sub_hi[dim] = new_hi;
        s->sub_len[dim] = new_size;
        box_changed = true;
    }
    if (box_changed) {
        s->bounds_changed = true;
        s->last_build_n = 0;  // neighbor.last_build_pos.clear()
    }
    if (!s->shear) return SOIL_OK;
    const double rate = s->shear_rate;
    const double lx = s->size[0], ly = s->size[1];
    const double dv = rate * ly;
    if (!s->shear_initialized) {
        *profile = true;
        s->shear_initialized = true;
    }
    const double raw = rate * s->dt * (double)s->deform_step * ly;
    const double xy = raw - lx * std::round(raw / lx);
    s->tilt[0] = xy;
    s->bvel[0] = dv;
    s->triclinic = true;
    s->bounds_changed = true;
    s->last_build_n = 0;  // neighbor.last_build_pos.clear()
    return SOIL_OK;
}

// The shear-only form the batch engine uses (batched systems have no
// orthogonal deform, so nothing can fail or need a remap).
bool deform_host(soil_sys* s) {
    bool profile = false;
    RemapSpec r;
    deform_step(s, &profile, &r);
    return profile;
}

double profile_center(const soil_sys* s) { return 0.5 * (s->blo[1] + s->bhi[1]); }

int phase_deform(soil_sys* s) {
    bool profile = false;
    RemapSpec r;
    TRY(deform_step(s, &profile, &r));
    launch_remap(s->st, s->nlocal, s->A, r);  // before the profile, which reads y
    if (profile) launch_shear_profile(s->st, s->nlocal, s->A, s->shear_rate, profile_center(s));
    return check_launch(s);
}

int phase_initial(soil_sys* s) {
    launch_initial(s->st, s->nlocal, s->A, s->dt, false, nullptr, nullptr, nullptr, 0, 0.0, nullptr,
                   nullptr);
    return check_launch(s);
}

// needs_rebuild (neighbor.rs:762-784) given the displacement answer.
bool needs_rebuild_with(const soil_sys* s, bool disp) {
    if (s->last_build_n != s->nlocal || s->nlocal == 0) return true;
    if (s->state == FULL_REBUILD) return true;
    if (s->every == 0) return disp;
    if (s->check) return s->steps_since_build >= s->every || disp;
    return s->steps_since_build >= s->every;
}

bool displacement_needed(const soil_sys* s) {
    if (s->last_build_n != s->nlocal || s->nlocal == 0) return false;
    if (s->every == 0) return true;
    if (s->check) return s->steps_since_build < s->every;
    return false;
}

int read_flags(soil_sys* s) {
    CK(cudaMemcpyAsync(s->hflags, s->dflags, sizeof(DevFlags), cudaMemcpyDeviceToHost, s->st));
    TRY(sync(s));
    if (s->hflags->fault & SOIL_SCAN_ERR)
        return fail(s->ctx, SOIL_ERR_CUDA, "a single-pass scan's look-back wait ran out");
    return SOIL_OK;
}

int phase_decide_rebuild(soil_sys* s) {
    // decide_rebuild, neighbor.rs:796-822 (run_if CommunicateOnly)
    if (s->state != COMMUNICATE_ONLY) return SOIL_OK;
    bool disp = false;
    if (displacement_needed(s)) {
        CK(cudaMemsetAsync(&s->dflags->rebuild, 0, 4, s->st));
        launch_disp_check(s->st, s->nlocal, s->A, s->lbx.p, s->lby.p, s->lbz.p,
                          displacement_threshold_sq(s), s->pbc_box, s->dflags, pbc_mask(s));
        TRY(check_launch(s));
        TRY(read_flags(s));
        disp = s->hflags->rebuild != 0;
    }
    if (needs_rebuild_with(s, disp)) s->state = FULL_REBUILD;
    else s->steps_since_build += 1;
    return SOIL_OK;
}

int phase_remove_ghosts(soil_sys* s) {
    if (s->state != FULL_REBUILD) return SOIL_OK;
    s->nghost = 0;
    return SOIL_OK;
}

int phase_zero_forces(soil_sys* s) {
    int zp[kMaxPlanes], nz;
    zero_planes_of(s, SOIL_COL_ZERO, zp, &nz);
    launch_zero_forces(s->st, s->nlocal + s->nghost, s->A, zp, nz);
    return check_launch(s);
}

int pbc_mask(const soil_sys* s) {
    int m = 0;
    for (int d = 0; d < 3; ++d)
        if (s->btype[d] == SOIL_BOUNDARY_PERIODIC) m |= 1 << d;
    return m;
}

// The locals with ghost images, in order, from the fold program of a border
// pass; their count stays on the device (reverse comm reads it there).
int fold_roots_build(soil_sys* s) {
    TRY(select_arrays(s));
    TRY(ensure(s, s->fold_roots, s->acap + 1));
    TRY(ensure(s, s->fold_nroots, 1));
    const uint64_t nl = s->nlocal;
    launch_fold_root_flags(s->st, nl, s->fold_start.p, s->sel_flag.p);
    launch_select(s->st, nl, s->sel_flag.p, s->sel_pos.p, s->scan_tmp.p, s->fold_roots.p);
    CK(cudaMemcpyAsync(s->fold_nroots.p, s->sel_pos.p + nl, 4, cudaMemcpyDeviceToDevice, s->st));
    TRY(check_launch(s));
    s->fold_roots_gen = s->border_gen;
    return SOIL_OK;
}

int phase_pbc(soil_sys* s) {
    if (s->state != FULL_REBUILD) return SOIL_OK;
    s->pk_valid = false;
    const int mask = pbc_mask(s);
    if (mask == 7 || s->nlocal == 0) {
        launch_pbc(s->st, s->nlocal, s->A, geom_of(s), s->bvel);
        return check_launch(s);
    }
    // slow path, domain.rs:641-662: wrap periodic axes, then remove the atoms
    // outside a fixed axis by swap_remove from the last index down
    TRY(select_arrays(s));
    BoundsArgs b;
    for (int d = 0; d < 3; ++d) {
        b.lo[d] = s->blo[d];
        b.hi[d] = s->bhi[d];
        b.size[d] = s->size[d];
    }
    b.periodic = mask;
    b.geom = geom_of(s);
    for (int d = 0; d < 3; ++d) b.bvel[d] = s->bvel[d];
    const uint64_t nl = s->nlocal;
    launch_pbc_bounded(s->st, nl, s->A, b, s->sel_flag.p);
    launch_select(s->st, nl, s->sel_flag.p, s->sel_pos.p, s->scan_tmp.p, s->sel_out.p);
    TRY(check_launch(s));
    CK(cudaMemcpyAsync(s->hword, s->sel_pos.p + nl, 4, cudaMemcpyDeviceToHost, s->st));
    TRY(sync(s));
    const uint64_t gone = s->hword[0];
    if (gone == 0) return SOIL_OK;
    std::vector<uint32_t> idx(gone);
    CK(cudaMemcpyAsync(idx.data(), s->sel_out.p, gone * 4, cudaMemcpyDeviceToHost, s->st));
    TRY(sync(s));
    // the layout reverse-order swap_remove leaves: slot r takes the then-last atom
    std::vector<uint32_t> at(nl);
    for (uint64_t i = 0; i < nl; ++i) at[i] = (uint32_t)i;
    uint64_t n = nl;
    for (uint64_t k = gone; k-- > 0;) {
        const uint64_t r = idx[k], last = n - 1;
        if (r != last) at[r] = at[last];
        n -= 1;
    }
    CK(cudaMemcpyAsync(s->sort_perm.p, at.data(), n * 4, cudaMemcpyHostToDevice, s->st));
    launch_perm_gather(s->st, n, s->sort_perm.p, s->A, s->B);
    if (s->slot_max) {
        const int o = s->slot_old;
        launch_slot_gather(s->st, n, s->sort_perm.p, s->slot_max, s->slot_width,
                           s->slot_tag[o].p, s->slot_val[o].p, s->slot_tag[1 - o].p,
                           s->slot_val[1 - o].p);
        s->slot_old = 1 - o;
    }
    TRY(check_launch(s));
    TRY(sync(s));  // the host copy of the permutation is released on return
    std::swap(s->A, s->B);
    s->colptrs_dirty = true;
    s->perm_valid = false;
    s->nlocal = n;
    s->state = FULL_REBUILD;
    return SOIL_OK;
}

// shrink_wrap (domain.rs:509-589): every step before pbc, shrink-wrapped
// axes take the locals' extent plus the padding.
int phase_shrink_wrap(soil_sys* s) {
    int mask = 0;
    for (int d = 0; d < 3; ++d)
        if (s->btype[d] == SOIL_BOUNDARY_SHRINK) mask |= 1 << d;
    if (!mask || s->nlocal == 0) return SOIL_OK;
    double padding;
    if (s->shrink_padding > 0.0) padding = s->shrink_padding;
    else if (s->domain_ghost_cutoff > 0.0) padding = s->domain_ghost_cutoff;
    else {
        const double mx = std::fmax(s->size[0], std::fmax(s->size[1], s->size[2]));
        padding = mx > 0.0 ? mx * 0.01 : 1.0;
    }
    TRY(ensure(s, s->ext, 6));
    CK(cudaMemsetAsync(s->ext.p, 0xFF, 3 * 8, s->st));
    CK(cudaMemsetAsync(s->ext.p + 3, 0, 3 * 8, s->st));
    launch_extent(s->st, s->nlocal, s->A, mask, s->ext.p);
    TRY(check_launch(s));
    unsigned long long key[6];
    static_assert(sizeof(key) <= kBorderStateWords * 4, "pinned word buffer too small");
    CK(cudaMemcpyAsync(s->hword, s->ext.p, sizeof(key), cudaMemcpyDeviceToHost, s->st));
    TRY(sync(s));
    std::memcpy(key, s->hword, sizeof(key));
    auto value = [](unsigned long long k) {
        const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double v;
        std::memcpy(&v, &b, 8);
        return v;
    };
    bool changed = false;
    for (int d = 0; d < 3; ++d) {
        if (!(mask & (1 << d))) continue;
        const double new_low = value(key[d]) - padding;
        const double new_high = value(key[3 + d]) + padding;
        const double tol = 1e-12;
        if (std::fabs(new_low - s->blo[d]) > tol || std::fabs(new_high - s->bhi[d]) > tol) {
            s->blo[d] = new_low;
            s->bhi[d] = new_high;
            s->sub_lo[d] = new_low;
            s->sub_hi[d] = new_high;
            changed = true;
        }
    }
    if (changed) {  // update_derived, domain.rs:171-177
        for (int d = 0; d < 3; ++d) {
            s->size[d] = s->bhi[d] - s->blo[d];
            s->sub_len[d] = s->sub_hi[d] - s->sub_lo[d];
        }
        s->bounds_changed = true;
    }
    return SOIL_OK;
}

// sort_atoms_by_bin (neighbor.rs:834-997), host part: grid recompute, sort
// counter, whether the sort runs (*run) and whether it is a periodic sort.
int sort_plan(soil_sys* s, bool* run, bool* periodic) {
    *run = false;
    if (s->bounds_changed) {
        if (s->cached_max_cutoff > 0.0) compute_bin_grid(s);  // recompute_bins
        s->bounds_changed = false;
        s->state = FULL_REBUILD;
    }
    s->sort_counter += 1;
    *periodic = s->sort_every > 0 && s->sort_counter >= s->sort_every;
    if (*periodic) s->sort_counter = 0;
    s->local_cells_valid = false;
    if (s->nlocal == 0 || s->total_cells == 0) return SOIL_OK;
    if (!*periodic && s->state != FULL_REBUILD) return SOIL_OK;
    *run = true;
    const uint64_t nc = s->total_cells;
    TRY(ensure(s, s->sort_cell, s->acap));
    TRY(ensure(s, s->sort_perm, s->acap));
    TRY(ensure(s, s->sorted_local_cell, s->acap));
    TRY(ensure(s, s->cell_counts, nc + 1, 0, 2 * nc + 64));
    TRY(ensure(s, s->cell_start, nc + 2, 0, 2 * nc + 64));
    TRY(ensure(s, s->cell_cursor, nc + 1, 0, 2 * nc + 64));
    TRY(ensure(s, s->scan_tmp, scan_temp_words(nc + s->acap + 2), 0,
               scan_temp_words(2 * nc + s->acap + 64)));
    TRY(ensure(s, s->sort_start, nc + 2, 0, 2 * nc + 64));
    return SOIL_OK;
}

// After the sort kernels ran: bookkeeping, and the column swap if the
// permutation was applied (periodic sorts of an identity order do not apply).
void sort_done(soil_sys* s, bool apply, bool periodic) {
    s->local_cells_valid = true;
    s->perm_valid = true;
    s->sorts += 1;
    if (apply) {
        std::swap(s->A, s->B);
        s->colptrs_dirty = true;
        // last_build_pos is re-saved by the neighbor build that follows every
        // permutation, so its permutation is not needed.
    }
    if (periodic && apply) {
        s->last_build_n = 0;
        s->state = FULL_REBUILD;
    }
}

int sort_run(soil_sys* s, bool periodic_sort, bool cells_done);
int phase_sort(soil_sys* s) {
    bool run, periodic_sort;
    TRY(sort_plan(s, &run, &periodic_sort));
    if (!run) return SOIL_OK;
    return sort_run(s, periodic_sort, false);
}

// The sort's kernels after sort_plan decided to run it; cells_done: the
// locals' cells are binned and counted already (launch_pbc_cells).
int sort_run(soil_sys* s, bool periodic_sort, bool cells_done) {
    s->pk_valid = false;
    const uint64_t nl = s->nlocal;
    const uint64_t nc = s->total_cells;
    if (!cells_done) {
        TRY(counts_zero(s, nc));
        launch_cells(s->st, 0, nl, s->A, grid_of(s), s->sort_cell.p, s->cell_counts.p);
    }
    TRY(scan_1p(s, s->cell_counts.p, s->sort_start.p, nc));
    launch_scatter_consume(s->st, nl, s->sort_cell.p, s->sort_start.p, s->cell_counts.p,
                           s->sort_perm.p);
    counts_consumed(s);
    launch_segsort(s->st, nc, s->sort_start.p, s->sort_perm.p);
    TRY(check_launch(s));

    bool apply = true;
    if (periodic_sort) {
        CK(cudaMemsetAsync(&s->dflags->not_identity, 0, 4, s->st));
        launch_identity_check(s->st, nl, s->sort_perm.p, s->dflags);
        TRY(check_launch(s));
        TRY(read_flags(s));
        apply = s->hflags->not_identity != 0;
    }
    if (apply) {
        // every column gathered through perm; ghosts (if any) are discarded by
        // the borders that always follows a permutation
        launch_perm_gather(s->st, nl, s->sort_perm.p, s->A, s->B, !s->forces_dead,
                           s->sort_cell.p, s->sorted_local_cell.p);
        if (s->slot_max) {  // slots move with their atoms
            const int o = s->slot_old;
            launch_slot_gather(s->st, nl, s->sort_perm.p, s->slot_max, s->slot_width,
                               s->slot_tag[o].p, s->slot_val[o].p, s->slot_tag[1 - o].p,
                               s->slot_val[1 - o].p);
            s->slot_old = 1 - o;
        }
        TRY(check_launch(s));
    } else {
        launch_permute_u32(s->st, nl, s->sort_perm.p, s->sort_cell.p, s->sorted_local_cell.p);
        TRY(check_launch(s));
    }
    sort_done(s, apply, periodic_sort);
    return SOIL_OK;
}

int phase_borders_defer(soil_sys* s, bool defer);
int phase_borders(soil_sys* s) { return phase_borders_defer(s, false); }

// borders, comm.rs:682-860 (single rank: all six swaps are self-sends).
// All three dims run on the device back to back; the host reads the swap
// totals once at the end.  If the ghosts did not fit, the arrays grow and the
// (deterministic) pass is repeated.  With `defer` (a fully periodic box, in a
// step whose neighbor build follows at once) the host does not wait: the
// totals are copied back behind the pass and read at the neighbor build's own
// synchronisation (borders_pending), whose kernels take the atom count from
// the device until then.
int phase_borders_defer(soil_sys* s, bool defer) {
    if (s->state != FULL_REBUILD) return SOIL_OK;
    s->borders_pending = false;  // a pass left pending by a failed step is replaced
    s->pk_valid = false;
    s->view_out = false;  // views are valid until the next rebuild
    s->nghost = 0;
    BorderDim bds[3];
    border_setup(s, bds);
    TRY(borders_reserve(s));
    const int mask = pbc_mask(s);
    defer = defer && mask == 7;
    uint32_t* hb = defer ? s->hword + kBorderStateWords : s->hword;
    const BorderPass bp = border_pass(bds);
    unsigned periodic_swaps = 0;
    for (int d = 0; d < 3; ++d)
        if (mask & (1 << d)) periodic_swaps |= 3u << (2 * d);
    const BorderCats cats = mask == 7 ? border_cats() : border_cats_masked(periodic_swaps);
    for (int attempt = 0; attempt < 4; ++attempt) {
        TRY(borders_arrays(s));
        SendPtrs send;
        for (int k = 0; k < kNumSwaps; ++k) send.p[k] = s->send[k].p;
        // With locals the passes write every word the host reads.
        if (s->nlocal == 0) CK(cudaMemsetAsync(s->bstate.p, 0, kBorderStateWords * 4, s->st));
        // A deferred pass with locals writes the words the host reads straight
        // into its (mapped) copy: no copy in the stream after the pass.
        const bool direct = defer && s->nlocal > 0;
        launch_borders(s->st, s->nlocal, s->acap, s->A, cats, bp, s->face_flags.p, s->bcount.p,
                       s->boff.p, s->bstate.p, s->ghost_root.p, s->ghost_chain.p, send,
                       s->fold_start.p, s->fold_list.p,
                       direct ? s->hword_dev + kBorderStateWords : nullptr);
        TRY(check_launch(s));
        if (!direct)
            CK(cudaMemcpyAsync(hb, s->bstate.p, kBorderStateWords * 4, cudaMemcpyDeviceToHost,
                               s->st));
        if (defer) {
            for (int d = 0; d < 3; ++d) s->pending_bds[d] = bds[d];
            s->borders_pending = true;
            return SOIL_OK;
        }
        TRY(sync(s));
        if (!hb[10]) break;
        if (attempt == 3) return fail(s->ctx, SOIL_ERR_CAPACITY, "ghost capacity did not converge");
        TRY(grow_atoms(s, (uint64_t)hb[3] + 1024, s->nlocal));  // hb[3]: atoms incl. all ghosts
    }
    TRY(borders_done(s, hb, bds));
    if (mask == 7) return SOIL_OK;
    // A swap with no neighbor (non-periodic axis) still packs the atoms at its
    // face, scanning the locals and the ghosts of the earlier axes
    // (pack_border_atoms, comm.rs:333-358), but nothing is received.
    TRY(select_arrays(s));
    for (int d = 0; d < 3; ++d) {
        if (mask & (1 << d)) continue;
        const uint64_t scan_end = s->swaps[2 * d].recv_start;  // atoms before this axis' swaps
        for (int sw = 0; sw < 2; ++sw) {
            const int k = 2 * d + sw;
            launch_face_flag(s->st, scan_end, s->A, bds[d].geom, d,
                             sw == 0 ? bds[d].thresh_lo : bds[d].thresh_hi, sw, s->sel_flag.p);
            launch_select(s->st, scan_end, s->sel_flag.p, s->sel_pos.p, s->scan_tmp.p, s->send[k].p);
            CK(cudaMemcpyAsync(s->sel_cnt.p + k, s->sel_pos.p + scan_end, 4, cudaMemcpyDeviceToDevice,
                               s->st));
        }
    }
    TRY(check_launch(s));
    uint32_t cnt[kNumSwaps];
    CK(cudaMemcpyAsync(cnt, s->sel_cnt.p, sizeof(cnt), cudaMemcpyDeviceToHost, s->st));
    TRY(sync(s));
    for (int d = 0; d < 3; ++d)
        if (!(mask & (1 << d)))
            for (int sw = 0; sw < 2; ++sw) s->swaps[2 * d + sw].send_count = cnt[2 * d + sw];
    return SOIL_OK;
}

// Face thresholds and image shifts of the three border dims (comm.rs:288-358,
// 736-761): lo swap shift +L, hi swap -L, the y shift carrying the tilt and
// the Lees–Edwards velocity jump.
void border_setup(const soil_sys* s, BorderDim bds[3]) {
    const double gc = s->domain_ghost_cutoff;
    for (int dim = 0; dim < 3; ++dim) {
        BorderDim& bd = bds[dim];
        bd.dim = dim;
        bd.triclinic = s->triclinic ? 1 : 0;
        bd.geom = geom_of(s);
        if (s->triclinic) {
            const double inflate = dim == 0 ? 1.0 + std::fabs(s->tilt[0]) / s->size[1] : 1.0;
            const double cut_l = (gc / s->size[dim]) * inflate;
            bd.thresh_lo = s->sub_lam_lo[dim] + cut_l;
            bd.thresh_hi = s->sub_lam_hi[dim] - cut_l;
        } else {
            bd.thresh_lo = s->sub_lo[dim] + gc;
            bd.thresh_hi = s->sub_hi[dim] - gc;
        }
        for (int sw = 0; sw < 2; ++sw) {
            // comm_setup periodic_swap (comm.rs:265-280): 0 without periodicity
            const double po = s->btype[dim] != SOIL_BOUNDARY_PERIODIC ? 0.0 : sw == 0 ? 1.0 : -1.0;
            double* sh = bd.shift[sw];
            if (dim == 0) { sh[0] = po * s->size[0]; sh[1] = 0.0; sh[2] = 0.0; }
            else if (dim == 1) { sh[0] = po * s->tilt[0]; sh[1] = po * s->size[1]; sh[2] = 0.0; }
            else { sh[0] = po * s->tilt[1]; sh[1] = po * s->tilt[2]; sh[2] = po * s->size[2]; }
            for (int d = 0; d < 3; ++d) bd.vshift[sw][d] = dim == 1 ? po * s->bvel[d] : 0.0;
            bd.swap_id[sw] = 2 * dim + sw;
        }
    }
}

// Capacity for this pass's ghosts: those of the last pass plus a margin.
int borders_reserve(soil_sys* s) {
    // ghosts of the last pass, or before any pass the count a uniform density
    // gives: locals x (prod (L_d + 2 gc) / prod L_d - 1)
    uint64_t g = s->last_nghost;
    if (g == 0 && s->nlocal) {
        double f = 1.0;
        for (int d = 0; d < 3; ++d)
            f *= (s->size[d] + 2.0 * s->domain_ghost_cutoff) / s->size[d];
        g = (uint64_t)((double)s->nlocal * (f - 1.0));
    }
    const uint64_t want = s->nlocal + g + g / 4 + 4096;
    TRY(grow_atoms(s, want, s->nlocal));
    return borders_arrays(s);
}

// Arrays of a borders pass at the current capacity: the fold program is
// written by the same pass, so it is sized for a full capacity of ghosts.
int borders_arrays(soil_sys* s) {
    const uint64_t cap = s->acap;
    const uint64_t nw = (s->nlocal + 31) / 32;
    TRY(ensure(s, s->bstate, kBorderStateWords));
    TRY(ensure(s, s->bcount, (kBorderCats + 1) * (nw + nw / 8192 + 1) + 1));
    TRY(ensure(s, s->boff, (kBorderCats + 1) * nw + 1));
    for (int k = 0; k < kNumSwaps; ++k) TRY(ensure(s, s->send[k], cap + 1));
    TRY(ensure(s, s->face_flags, cap + 1));
    TRY(ensure(s, s->fold_start, s->nlocal + 2));
    TRY(ensure(s, s->fold_list, cap + 1));
    return SOIL_OK;
}

// Swap records and ghost count from a finished pass (hb: its border state),
// and room for the reverse-comm fold program.
int borders_done(soil_sys* s, const uint32_t* hb, const BorderDim bds[3]) {
    for (int dim = 0; dim < 3; ++dim) {
        const uint64_t recv_lo = hb[dim], n_lo = hb[4 + dim], n_hi = hb[7 + dim];
        for (int sw = 0; sw < 2; ++sw) {
            SwapHost& h = s->swaps[2 * dim + sw];
            h.recv_start = sw == 0 ? recv_lo : recv_lo + n_lo;
            h.recv_count = sw == 0 ? n_lo : n_hi;
            h.send_count = h.recv_count;
            for (int d = 0; d < 3; ++d) {
                h.off[d] = bds[dim].shift[sw][d];
                h.voff[d] = bds[dim].vshift[sw][d];
            }
        }
    }
    s->nghost = (uint64_t)hb[3] - s->nlocal;
    s->last_nghost = s->nghost;
    s->border_gen += 1;
    s->nswaps = kNumSwaps;
    // A local has images on both sides of a periodic dim only when the two
    // face slabs overlap; otherwise it has at most 7 images.
    const int mask = pbc_mask(s);
    s->few_images = true;
    for (int d = 0; d < 3; ++d)
        if ((mask & (1 << d)) && bds[d].thresh_lo > bds[d].thresh_hi) s->few_images = false;
    return SOIL_OK;
}

SwapConst swap_const(const soil_sys* s) {
    SwapConst sc;
    for (int k = 0; k < kNumSwaps; ++k)
        for (int d = 0; d < 3; ++d) {
            sc.off[k][d] = s->swaps[k].off[d];
            sc.voff[k][d] = s->swaps[k].voff[d];
        }
    return sc;
}

int forward_comm(soil_sys* s, bool zero_ghost_force) {
    int fp[kMaxPlanes], nf;
    zero_planes_of(s, SOIL_COL_FORWARD, fp, &nf);
    launch_forward(s->st, s->nlocal, s->nghost, s->A, s->ghost_root.p, s->ghost_chain.p,
                   swap_const(s), fp, nf, zero_ghost_force);
    return check_launch(s);
}

int phase_forward_comm(soil_sys* s) {
    if (s->state != COMMUNICATE_ONLY) return SOIL_OK;
    return forward_comm(s, false);
}

int build_in_lists(soil_sys* s) {
    const uint64_t total = s->nlocal + s->nghost;
    TRY(ensure(s, s->in_count, total + 1, 0, s->acap + 1));
    TRY(ensure(s, s->in_start, total + 2, 0, s->acap + 2));
    TRY(ensure(s, s->in_cursor, total + 1, 0, s->acap + 1));
    TRY(ensure(s, s->in_list, s->npairs + 1, 0, pair_room(s->npairs)));
    TRY(ensure(s, s->scan_tmp, scan_temp_words(total + 2)));
    CK(cudaMemsetAsync(s->in_count.p, 0, total * 4, s->st));
    s->in_zero = 0;  // left holding the counts
    launch_in_count(s->st, s->nlocal, s->offsets.p, s->indices.p, s->in_count.p);
    TRY(scan_1p(s, s->in_count.p, s->in_start.p, total));
    CK(cudaMemcpyAsync(s->in_cursor.p, s->in_start.p, total * 4, cudaMemcpyDeviceToDevice, s->st));
    launch_in_scatter(s->st, s->nlocal, s->offsets.p, s->indices.p, s->in_cursor.p, s->in_list.p);
    TRY(ensure(s, s->in_split, total + 1, 0, s->acap + 1));
    launch_segsort_split(s->st, total, s->in_start.p, s->in_list.p, s->in_split.p);
    TRY(check_launch(s));
    s->in_lists_valid = true;
    s->split_valid = true;
    return SOIL_OK;
}

// The built-in consumer's grouped partner sequences (from the CSR, the
// transposed lists and the fold program): one entry per (atom, contribution),
// 2 per pair with newton.
int build_seq(soil_sys* s) {
    const uint64_t total = s->nlocal + s->nghost, nl = s->nlocal;
    const uint64_t room = 2 * pair_room(s->npairs);
    TRY(ensure(s, s->seq_cnt, total + 1, 0, s->acap + 1));
    TRY(ensure(s, s->grp_cnt, nl + 1, 0, s->acap + 1));
    TRY(ensure(s, s->grp_start, nl + 2, 0, s->acap + 2));
    TRY(ensure(s, s->seq, 2 * s->npairs + 1, 0, room));
    TRY(ensure(s, s->seq_owner, 2 * s->npairs + 1, 0, room));
    TRY(ensure(s, s->scan_tmp, scan_temp_words(total + 2)));
    SeqArgs q;
    q.nlocal = nl;
    q.ntotal = total;
    q.newton = s->newton ? 1 : 0;
    q.offsets = s->offsets.p;
    q.indices = s->indices.p;
    q.in_start = s->in_start.p;
    q.in_list = s->in_list.p;
    q.fold_start = s->fold_start.p;
    q.fold_list = s->fold_list.p;
    launch_seq_count(s->st, q, s->seq_cnt.p, s->grp_cnt.p);
    TRY(scan_1p(s, s->grp_cnt.p, s->grp_start.p, nl));
    launch_seq_fill(s->st, q, s->grp_start.p, s->seq.p, s->seq_owner.p);
    TRY(check_launch(s));
    s->seq_valid = true;
    return SOIL_OK;
}

// Whether the grouped consumer serves this system: the built-in consumer,
// and a ghost layout in which no local has images on both sides of a dim
// (at most 7 images per root, what the sequences' owner byte encodes).
bool seq_consumer(const soil_sys* s) { return builtin_consumer(s) && s->few_images; }

// Whether the one-thread-per-root consumer kernels read the packed records
// (SOIL_PACKED=1; read at each call).  Off by default: on 4M atoms the
// records' 40 B per atom and step in the integration pass cost more than
// the walks gain from one 32-byte load per partner.
bool packed_on() {
    const char* env = std::getenv("SOIL_PACKED");
    return env && std::atoi(env) == 1;
}

// The packed records, current for every local and ghost: allocated with the
// atom capacity and packed from the columns when stale (each rebuild step and
// host write marks them so); from then on the integration pass and forward
// comm keep them current through AtomCols::pk.
int pk_ready(soil_sys* s) {
    if (!packed_on()) {
        s->A.pk = s->B.pk = nullptr;
        s->pk_valid = false;
        return SOIL_OK;
    }
    const double* old = s->pk.p;
    TRY(ensure(s, s->pk, 4 * s->acap));
    if (s->pk.p != old) s->pk_valid = false;
    if (reinterpret_cast<uintptr_t>(s->pk.p) % 32)
        return fail(s->ctx, SOIL_ERR_CUDA, "packed records: allocation not 32-byte aligned");
    const int rp = s->cols[s->radius_col].plane0;
    s->A.pk = s->B.pk = s->pk.p;
    s->A.pkrad = s->A.planes[rp];
    s->B.pkrad = s->B.planes[rp];
    if (!s->pk_valid) {
        launch_pack(s->st, s->nlocal + s->nghost, s->A,
                    s->A.planes[s->cols[s->radius_col].plane0], s->pk.p);
        TRY(check_launch(s));
        s->pk_valid = true;
    }
    return SOIL_OK;
}

ForceArgs consumer_args(const soil_sys* s) {
    ForceArgs p;
    p.c = s->A;
    p.q.rad = s->A.planes[s->cols[s->radius_col].plane0];
    p.q.K = s->harmonic_k;
    p.q.nlocal = s->nlocal;
    p.q.grp_start = s->grp_start.p;
    p.q.cnt = s->seq_cnt.p;
    p.q.seq = s->seq.p;
    p.q.owner = s->seq_owner.p;
    p.q.fold_start = s->fold_start.p;
    p.q.fold_list = s->fold_list.p;
    p.q.pk = s->pk_valid ? s->pk.p : nullptr;
    zero_planes_of(s, SOIL_COL_REVERSE, p.rev.idx, &p.rev.n);
    return p;
}

ForceCsr csr_args(const soil_sys* s) {
    ForceCsr q;
    q.order = nullptr;
    q.rad = s->A.planes[s->cols[s->radius_col].plane0];
    q.K = s->harmonic_k;
    q.nlocal = s->nlocal;
    q.newton = s->newton ? 1 : 0;
    q.offsets = s->offsets.p;
    q.indices = s->indices.p;
    q.in_start = s->in_start.p;
    q.in_list = s->in_list.p;
    q.in_split = s->in_split.p;
    q.fold_start = s->fold_start.p;
    q.fold_list = s->fold_list.p;
    q.pk = s->pk_valid ? s->pk.p : nullptr;
    return q;
}

// The CSR walk's per-block root order when SOIL_ROOT_ORDER=1 (built once per
// set of lists), else index order: measured on 4M atoms, ordering roots by
// work gave each warp more even trips but scattered the roots' own reads and
// writes, and the walk ran slower.
int csr_with_order(soil_sys* s, ForceCsr* q) {
    if (!s->split_valid) {  // transposed lists sorted elsewhere (a batch)
        const uint64_t total = s->nlocal + s->nghost;
        TRY(ensure(s, s->in_split, total + 1, 0, s->acap + 1));
        launch_in_split(s->st, total, s->in_start.p, s->in_list.p, s->in_split.p);
        TRY(check_launch(s));
        s->split_valid = true;
    }
    *q = csr_args(s);
    const char* env = std::getenv("SOIL_ROOT_ORDER");
    if (!env || std::atoi(env) != 1) return SOIL_OK;
    if (!s->order_valid) {
        TRY(ensure(s, s->root_order, s->nlocal + 1, 0, s->acap + 1));
        launch_root_order(s->st, *q, s->root_order.p);
        TRY(check_launch(s));
        s->order_valid = true;
    }
    q->order = s->root_order.p;
    return SOIL_OK;
}

// Whether the consumer kernel folds reverse comm into itself (newton): the
// CSR walk always, the grouped-sequence kernels when they serve the system.
bool consumer_folds(const soil_sys* s) {
    if (s->hook || !builtin_consumer(s) || !s->newton) return false;
    const int v = force_variant();
    if (v == SOIL_FORCE_GATHER) return false;
    return v == SOIL_FORCE_CSR || seq_consumer(s);
}

// The built-in consumer; with fold (newton), reverse comm of the forces and
// #[reverse] planes is done in the same kernel.
int launch_consumer(soil_sys* s, bool fold) {
    if (!s->in_lists_valid) TRY(build_in_lists(s));
    const int variant = force_variant();
    if (variant != SOIL_FORCE_GATHER) TRY(pk_ready(s));
    if (variant == SOIL_FORCE_CSR) {
        PlaneList rev;
        zero_planes_of(s, SOIL_COL_REVERSE, rev.idx, &rev.n);
        ForceCsr q;
        TRY(csr_with_order(s, &q));
        launch_force_csr(s->st, q, s->A, rev, fold);
        return check_launch(s);
    }
    if (!seq_consumer(s) || variant == SOIL_FORCE_GATHER) {
        launch_harmonic(s->st, s->nlocal, s->nlocal + s->nghost, s->A,
                        s->A.planes[s->cols[s->radius_col].plane0], s->harmonic_k,
                        s->newton ? 1 : 0, s->offsets.p, s->indices.p, s->in_start.p,
                        s->in_list.p);
        return check_launch(s);
    }
    if (!s->seq_valid) TRY(build_seq(s));
    launch_force_seq(s->st, consumer_args(s), fold, variant);
    return check_launch(s);
}

// bin_neighbor_list (neighbor.rs:1013-1319), host part: the CommState
// transition, save_build_positions bookkeeping (neighbor.rs:669-690; the local
// cutoff radii never change after setup, so their min/max are cached there),
// the uniform-cutoff decision (neighbor_params, a function of those constants
// only) and room for the build.
void neighbor_params(soil_sys* s) {
    s->cached_min_skin = s->cut_min_local;
    if (std::fabs(s->cut_max_local - s->cut_min_local) < 1e-15) {
        const double cutoff = 2.0 * s->cut_min_local * s->skin_fraction;
        s->has_uniform = true;
        s->uniform_cut_sq = cutoff * cutoff;
    } else {
        s->has_uniform = false;
    }
}

int neighbor_plan(soil_sys* s) {
    s->state = COMMUNICATE_ONLY;
    const uint64_t nl = s->nlocal;
    TRY(ensure(s, s->lbx, s->acap));
    TRY(ensure(s, s->lby, s->acap));
    TRY(ensure(s, s->lbz, s->acap));
    s->last_build_n = nl;
    s->steps_since_build = 0;
    neighbor_params(s);
    const uint64_t nc = s->total_cells;
    TRY(ensure(s, s->atom_cell, s->acap));
    TRY(ensure(s, s->sorted_atoms, s->acap));
    TRY(ensure(s, s->asi, s->acap));
    TRY(ensure(s, s->rowcount, s->acap));
    TRY(ensure(s, s->offsets, s->acap + 2));
    TRY(ensure(s, s->sp, s->acap));
    if (s->filter == SOIL_FILTER_FP32_RECHECK) TRY(ensure(s, s->spf, s->acap));
    TRY(ensure(s, s->row_slots, (uint64_t)nl * kRowSlots + 1));
    TRY(ensure(s, s->cell_counts, nc + 1, 0, 2 * nc + 64));
    TRY(ensure(s, s->cell_start, nc + 2, 0, 2 * nc + 64));
    TRY(ensure(s, s->cell_cursor, nc + 1, 0, 2 * nc + 64));
    TRY(ensure(s, s->scan_tmp, scan_temp_words(nc + s->acap + 2), 0,
               scan_temp_words(2 * nc + s->acap + 64)));
    TRY(ensure(s, s->ghost_tmp, s->acap));
    return SOIL_OK;
}

// The stencil as segments of consecutive cells in scan order (the own cell
// first); false when there are too many for the staged pair count (or
// SOIL_PAIRS_STAGED=0), which then scans from global memory.
bool pair_segments(const std::vector<int32_t>& sten, bool has_self, bool newton, PairSegs* sg) {
    const char* env = std::getenv("SOIL_PAIRS_STAGED");
    if (!env || std::atoi(env) == 0) return false;  // measured slower: off unless asked
    sg->n = 0;
    sg->own = has_self ? 1 : 0;
    if (has_self) {
        sg->off[0] = 0;
        sg->len[0] = 1;
        sg->n = 1;
    }
    for (const int32_t off : sten) {
        if (!newton && off == 0) continue;  // the own cell is scanned first
        const int k = sg->n - 1;
        if (k >= sg->own && sg->off[k] + sg->len[k] == off) {
            sg->len[k] += 1;
            continue;
        }
        if (sg->n == kMaxPairSegs) return false;
        sg->off[sg->n] = off;
        sg->len[sg->n] = 1;
        sg->n += 1;
    }
    sg->nrun = 0;
    for (int k = 0; k < sg->n; ++k) {
        const int r = sg->nrun - 1;
        if (r >= 0 && sg->roff[r] + sg->rlen[r] == sg->off[k]) {
            sg->rlen[r] += sg->len[k];
        } else {
            sg->roff[sg->nrun] = sg->off[k];
            sg->rlen[sg->nrun] = sg->len[k];
            sg->nrun += 1;
        }
        sg->run[k] = sg->nrun - 1;
    }
    return true;
}

// Margin of the FP32 prefilter: FP32 coordinates are relative to the box
// corner and M bounds their magnitude.
float pair_eps(const soil_sys* s) {
    double M = 0.0;
    for (int d = 0; d < 3; ++d) M = std::fmax(M, s->size[d]);
    M += 2.0 * s->domain_ghost_cutoff + std::fabs(s->tilt[0]) + 4.0 * s->cached_max_cutoff;
    return (float)(1e-6 * (1.0 + s->cached_max_cutoff) + 4e-7 * M);
}

int phase_neighbor(soil_sys* s) {
    if (s->state != FULL_REBUILD) return SOIL_OK;
    TRY(neighbor_plan(s));
    const uint64_t nl = s->nlocal;
    // Until a deferred border pass is read back, the atom count is the
    // device's (bstate word 3) and `total` the capacity that bounds it.
    const bool pend = s->borders_pending;
    uint64_t total = pend ? s->acap : s->nlocal + s->nghost;
    const uint32_t* n_dev = pend ? s->bstate.p + 3 : nullptr;
    const uint64_t nc = s->total_cells;
    const bool fp32 = s->filter == SOIL_FILTER_FP32_RECHECK;
    TRY(counts_zero(s, nc));
    const Grid gr = grid_of(s);
    const bool after_sort = s->local_cells_valid;
    if (after_sort)  // reuse the sort's local cells (neighbor.rs:1049-1066)
        launch_cells_reuse(s->st, nl, total, s->A, gr, s->sorted_local_cell.p, s->atom_cell.p,
                           s->cell_counts.p, n_dev);
    else
        launch_cells(s->st, 0, total, s->A, gr, s->atom_cell.p, s->cell_counts.p, n_dev);
    s->local_cells_valid = false;
    TRY(scan_1p(s, s->cell_counts.p, s->cell_start.p, nc));
    if (after_sort) {
        // the locals are in bin order already: only the ghosts are sorted
        const bool zeroed =
            launch_place_bins(s->st, nl, total, nc, n_dev, s->atom_cell.p, s->cell_start.p,
                              s->sort_start.p, s->cell_counts.p, s->ghost_tmp.p,
                              s->sorted_atoms.p);
        s->counts_clean = zeroed ? nc : 0;  // else the locals' counts remain
    } else {
        launch_scatter_consume(s->st, total, s->atom_cell.p, s->cell_start.p, s->cell_counts.p,
                               s->sorted_atoms.p, n_dev);
        counts_consumed(s);
        launch_segsort(s->st, nc, s->cell_start.p, s->sorted_atoms.p);
    }
    BuildPos bpos;  // save_build_positions (neighbor.rs:669-690) in the same pass
    bpos.x = s->lbx.p;
    bpos.y = s->lby.p;
    bpos.z = s->lbz.p;
    bpos.nlocal = nl;
    launch_sorted_views(s->st, total, s->sorted_atoms.p, s->A, s->asi.p, s->sp.p,
                        fp32 ? s->spf.p : nullptr, s->blo, bpos, n_dev, s->has_uniform,
                        s->dflags);  // also clears the counters of the pair passes
    const std::vector<int32_t>& sten = s->newton ? s->stencil_fwd : s->stencil;
    const std::vector<int32_t> runs = stencil_runs(sten, s->newton);
    const int32_t* old_stencil = s->d_stencil.p;
    TRY(ensure(s, s->d_stencil, runs.size() + 1));
    if (!runs.empty() && (s->d_stencil.p != old_stencil || runs != s->stencil_on_device)) {
        // pageable source: the copy completes before cudaMemcpyAsync returns
        CK(cudaMemcpyAsync(s->d_stencil.p, runs.data(), runs.size() * 4, cudaMemcpyHostToDevice, s->st));
        s->stencil_on_device = runs;
    }
    PairParams p;
    p.atom_cell = s->atom_cell.p;
    p.atom_sorted_idx = s->asi.p;
    p.bin_start = s->cell_start.p;
    p.sorted_atoms = s->sorted_atoms.p;
    p.sp = s->sp.p;
    p.spf = s->spf.p;
    p.stencil = s->d_stencil.p;
    p.nstencil = (int)(runs.size() / 2);
    p.ncells = (uint32_t)nc;
    p.nlocal = nl;
    p.row_slots = kRowSlots;
    p.has_self = s->stencil_self ? 1 : 0;
    p.newton = s->newton ? 1 : 0;
    p.uniform = s->has_uniform ? 1 : 0;
    p.filter = s->filter;
    p.cut_sq = s->uniform_cut_sq;
    p.sf_sq = s->skin_fraction * s->skin_fraction;
    p.sf = s->skin_fraction;
    p.eps32 = pair_eps(s);
    // candidates, rechecked and error are adjacent: one clear (the sorted
    // views cleared them when there were atoms)
    static_assert(offsetof(DevFlags, error) == offsetof(DevFlags, candidates) + 16, "DevFlags layout");
    if (total == 0) CK(cudaMemsetAsync(&s->dflags->candidates, 0, 20, s->st));
    s->in_lists_valid = false;
    s->seq_valid = false;
    s->order_valid = false;
    // The transposed lists serve the built-in consumer and any force hook:
    // the pair passes build them too (pass 1 counts each partner's entries,
    // pass 2 places every row in its partners' lists), then a per-atom sort
    // restores ascending order.
    const bool with_in = builtin_consumer(s) || s->hook;
    p.in_count = nullptr;
    p.in_start = nullptr;
    p.in_list = nullptr;
    p.pre_ranges = pairs_pre_ranges();
    uint64_t in_zero = 0;  // in_count[0, in_zero) is zero already
    const uint64_t in_range = total;  // the counts pass 1 may write and the scan reads
    if (with_in) {
        TRY(ensure(s, s->in_count, total + 1, 0, s->acap + 1));
        TRY(ensure(s, s->in_start, total + 2, 0, s->acap + 2));
        in_zero = s->in_zero_at == s->in_count.p ? s->in_zero : 0;
        if (in_zero < total)
            CK(cudaMemsetAsync(s->in_count.p + in_zero, 0, (total - in_zero) * 4, s->st));
        s->in_zero = 0;  // counted into now; zero again once pass 2 has consumed it
        s->in_zero_at = s->in_count.p;
        p.in_count = s->in_count.p;
    }
    PairSegs sg;
    if (pair_segments(sten, s->stencil_self, s->newton, &sg))
        launch_pair_count_staged(s->st, p, sg, s->rowcount.p, s->row_slots.p, s->dflags);
    else
        launch_pair_count(s->st, p, s->rowcount.p, s->row_slots.p, s->dflags);
    if (with_in) TRY(scan_pair(s, s->rowcount.p, s->offsets.p, nl, s->in_count.p, s->in_start.p, total));
    else TRY(scan_1p(s, s->rowcount.p, s->offsets.p, nl));
    if (!s->ev_counts) CK(cudaEventCreateWithFlags(&s->ev_counts, cudaEventDisableTiming));
    // Pass 2 goes in before the host reads the pair total, into the arrays it
    // has: the stream stays busy while the host waits for the counts, which
    // pass 2 itself writes to the host's words.  The guard lets it run only
    // when the total fits (and nothing failed); else it is launched again
    // below, into grown arrays.  (The transposed lists hold one entry per
    // pair, so one total bounds both arrays.)
    if (with_in) {
        TRY(ensure(s, s->in_split, total + 1, 0, s->acap + 1));
        p.in_start = s->in_start.p;
        p.in_list = s->in_list.p;
    }
    FillGuard guard;
    guard.total = s->offsets.p + nl;
    guard.cap = s->indices.cap;
    if (with_in && s->in_list.cap < guard.cap) guard.cap = s->in_list.cap;
    guard.err = &s->dflags->error;
    guard.pub_total = s->hword_dev;
    guard.flags = s->dflags;
    guard.pub_flags = s->hflags_dev;
    const bool early = s->indices.p && (!with_in || s->in_list.p) && nl > 0;
    if (early) {
        launch_pair_fill(s->st, p, s->rowcount.p, s->row_slots.p, s->offsets.p, s->indices.p,
                         guard);
        CK(cudaEventRecord(s->ev_counts, s->st));
        if (with_in)
            launch_segsort_split(s->st, total, s->in_start.p, s->in_list.p, s->in_split.p, &guard);
    } else {
        CK(cudaMemcpyAsync(&s->hword[0], s->offsets.p + nl, 4, cudaMemcpyDeviceToHost, s->st));
        CK(cudaMemcpyAsync(s->hflags, s->dflags, sizeof(DevFlags), cudaMemcpyDeviceToHost, s->st));
        CK(cudaEventRecord(s->ev_counts, s->st));
    }
    TRY(check_launch(s));
    CK(cudaEventSynchronize(s->ev_counts));
    if (s->hflags->fault & SOIL_SCAN_ERR)
        return fail(s->ctx, SOIL_ERR_CUDA, "a single-pass scan's look-back wait ran out");
    if (pend) {  // the deferred border pass, now read back
        s->borders_pending = false;
        const uint32_t* hb = s->hword + kBorderStateWords;
        if (hb[10]) {
            // The ghosts did not fit: grow, then repeat the border pass and
            // this build with the host reading the ghost counts first.
            TRY(grow_atoms(s, (uint64_t)hb[3] + 1024, s->nlocal));
            s->state = FULL_REBUILD;
            TRY(phase_borders_defer(s, false));
            return phase_neighbor(s);
        }
        TRY(borders_done(s, hb, s->pending_bds));
        total = s->nlocal + s->nghost;
    }
    const uint64_t np = s->hword[0];
    if (s->hflags->error & SOIL_PAIRS_ERR_STAGING)
        return fail(s->ctx, SOIL_ERR_CUDA, "pair build: a shared-memory staging wait ran out");
    if (s->hflags->error)
        return fail(s->ctx, SOIL_ERR_INVALID, "neighbor stencil left the bin grid (atom outside the ghost layers)");
    if (!early || np + 1 > guard.cap) {  // the early pass did not run: again, into room for np
        TRY(ensure(s, s->indices, np + 1, 0, pair_room(np)));
        if (with_in) {
            TRY(ensure(s, s->in_list, np + 1, 0, pair_room(np)));
            p.in_list = s->in_list.p;
        }
        launch_pair_fill(s->st, p, s->rowcount.p, s->row_slots.p, s->offsets.p, s->indices.p);
        if (with_in)
            launch_segsort_split(s->st, total, s->in_start.p, s->in_list.p, s->in_split.p);
        TRY(check_launch(s));
    }
    s->npairs = np;
    s->rebuilds += 1;
    if (with_in) {
        s->in_lists_valid = true;
        s->split_valid = true;
        s->in_zero = in_zero > in_range ? in_zero : in_range;  // pass 2 took every count back
    }
    // the grouped sequences are built when a consumer kernel first needs them
    return SOIL_OK;
}

int make_view(soil_sys* s, soil_dev_view* v) {
    std::memset(v, 0, sizeof(*v));
    s->pk_valid = false;  // the holder of a view may write any column
    TRY(update_colptrs(s));
    v->nlocal = s->nlocal;
    v->nghost = s->nghost;
    v->npairs = s->npairs;
    v->stride = s->acap;
    v->x = s->A.x; v->y = s->A.y; v->z = s->A.z;
    v->vx = s->A.vx; v->vy = s->A.vy; v->vz = s->A.vz;
    v->fx = s->A.fx; v->fy = s->A.fy; v->fz = s->A.fz;
    v->mass = s->A.mass;
    v->inv_mass = s->A.inv_mass;
    v->cutoff_radius = s->A.cut;
    v->tag = s->A.tag;
    v->neighbor_offsets = s->offsets.p;
    v->neighbor_indices = s->indices.p;
    v->ncolumns = (int32_t)s->cols.size();
    v->newton = s->newton ? 1 : 0;
    v->columns = s->d_colptrs.p;
    v->stream = (void*)s->st;
    v->in_start = s->in_lists_valid ? s->in_start.p : nullptr;
    v->in_list = s->in_lists_valid ? s->in_list.p : nullptr;
    v->origin = s->A.origin;
    v->fold_start = s->fold_start.p;
    v->fold_list = s->fold_list.p;
    v->ghost_root = s->ghost_root.p;
    if (s->slot_max) {
        const int o = s->slot_old;
        v->slot_max = s->slot_max;
        v->slot_width = s->slot_width;
        v->slot_old_tag = s->slot_tag[o].p;
        v->slot_old_val = s->slot_val[o].p;
        v->slot_new_tag = s->slot_tag[1 - o].p;
        v->slot_new_val = s->slot_val[1 - o].p;
    }
    return SOIL_OK;
}

int phase_force(soil_sys* s) {
    if (s->hook) {
        if (!s->in_lists_valid && s->npairs + s->nlocal > 0) TRY(build_in_lists(s));
        soil_dev_view v;
        TRY(make_view(s, &v));
        int r = s->hook(&v, s->hook_user);
        if (r != 0) return fail(s->ctx, SOIL_ERR_INVALID, "force hook returned %d", r);
        if (s->slot_max) s->slot_old = 1 - s->slot_old;  // this step's slots are next step's old
        return check_launch(s);
    }
    if (!builtin_consumer(s)) return SOIL_OK;
    return launch_consumer(s, false);
}

// Whether a step's reverse comm can change anything.  Without a consumer or
// a force hook nothing writes a force after the step's zeroing, so every
// ghost carries its root's +0 (borders copy it, forward comm zeroes it) and
// every fold adds +0 to +0; with no #[reverse] column nothing else is
// folded.  Such a step skips the pass (the per-phase entry point still runs
// it).
bool reverse_needed(const soil_sys* s) {
    if (builtin_consumer(s) || s->hook) return true;
    int rp[kMaxPlanes], nr;
    zero_planes_of(s, SOIL_COL_REVERSE, rp, &nr);
    return nr > 0;
}

int phase_reverse_comm(soil_sys* s) {
    // reverse_send_force, comm.rs:938-1024: rounds last to first, lo then hi;
    // each root's image tree in fold order, over the roots that have images
    if (!s->newton) return SOIL_OK;
    if (s->nswaps == 0 || s->nghost == 0) return SOIL_OK;
    int rp[kMaxPlanes], nr;
    zero_planes_of(s, SOIL_COL_REVERSE, rp, &nr);
    // A border pass folded once (every-step rebuilds) walks every local's fold
    // program; from its second fold on, the list of the locals that have
    // images is built once and walked instead.
    if (s->fold_roots_gen != s->border_gen && s->reverse_gen == s->border_gen)
        TRY(fold_roots_build(s));
    if (s->fold_roots_gen == s->border_gen)
        launch_reverse_fold_roots(s->st, s->nlocal, s->nghost, s->fold_nroots.p, s->fold_roots.p,
                                  s->fold_start.p, s->fold_list.p, s->A, rp, nr);
    else
        launch_reverse_fold(s->st, s->nlocal, s->fold_start.p, s->fold_list.p, s->A, rp, nr);
    s->reverse_gen = s->border_gen;
    return check_launch(s);
}

int phase_final(soil_sys* s) {
    launch_final(s->st, s->nlocal, s->A, s->dt);
    s->steps_done += 1;
    return check_launch(s);
}

// Forward comm may run inside the integration pass: the step starts with
// valid lists and ghosts (CommunicateOnly), and nothing between the
// integration and forward comm moves atoms or changes the box or the swap
// offsets (no deform, shear or shrink-wrap).
bool fused_forward_allowed(const soil_sys* s) {
    if (s->state != COMMUNICATE_ONLY || s->nghost == 0 || s->nswaps == 0) return false;
    if (s->shear || has_axis_deform(s)) return false;
    for (int d = 0; d < 3; ++d)
        if (s->btype[d] == SOIL_BOUNDARY_SHRINK) return false;
    return true;
}

// ... and SOIL_FWD_FUSED=1 puts it in the pass of soil_step's
// launch-per-phase steps.  Off by default: it measured slower there (most
// warps hold a lane whose root has images, and stall on its scattered ghost
// writes; k_forward writes the ghosts coalesced).  The resident steps always
// fuse it, which saves them a grid barrier.
bool fused_forward_ok(const soil_sys* s) {
    const char* env = std::getenv("SOIL_FWD_FUSED");
    if (!env || std::atoi(env) == 0) return false;
    return fused_forward_allowed(s);
}

// What the integration pass of a step decided, for the rest of the step.
struct StepPlan {
    bool overwrite;   // the built-in consumer overwrites every force
    bool fused_zero;  // forces zeroed in the integration pass (and forward comm)
    bool check;       // the displacement check ran in the integration pass
    bool fwd_fused;   // forward comm ran in the integration pass
    int nz;           // #[zero] planes
    // pbc (and, when the sort is due, its binning) ran in the integration
    // pass of a step that rebuilds for certain; sort_plan's answers
    bool pbc_done = false, sort_due = false, periodic_sort = false;
};

StepPlan plan_step(const soil_sys* s) {
    StepPlan p;
    p.overwrite = builtin_consumer(s);
    int zp[kMaxPlanes];
    zero_planes_of(s, SOIL_COL_ZERO, zp, &p.nz);
    p.fused_zero = !p.overwrite && p.nz == 0;
    p.check = s->state == COMMUNICATE_ONLY && displacement_needed(s);
    p.fwd_fused = fused_forward_ok(s);
    return p;
}

FwdArgs fwd_args(const soil_sys* s, bool fused_zero) {
    FwdArgs fw;
    fw.fold_start = s->fold_start.p;
    fw.fold_list = s->fold_list.p;
    fw.chain = s->ghost_chain.p;
    fw.sc = swap_const(s);
    zero_planes_of(s, SOIL_COL_FORWARD, fw.fwd.idx, &fw.fwd.n);
    fw.zero_ghost_force = fused_zero ? 1 : 0;
    return fw;
}

// The first part of a timestep: deform, then the integration pass with its
// fused displacement check (and forward comm).
int step_integrate(soil_sys* s, StepPlan* out) {
    const bool profile_now = s->deform_initialized && s->shear && !s->shear_initialized;
    if (profile_now && s->pending_final) {
        launch_final(s->st, s->nlocal, s->A, s->dt);
        s->pending_final = false;
    }
    timer_begin(s, T_INTEGRATE);
    TRY(phase_deform(s));
    StepPlan p = plan_step(s);
    if (p.check) CK(cudaMemsetAsync(&s->dflags->rebuild, 0, 4, s->st));
    // A step that rebuilds whatever its displacement check would say (lists
    // due, a box that moved), in a fully periodic box: pbc, and the sort's
    // binning when it falls due, ride on the integration pass.  decide_rebuild
    // has nothing left to decide, and the sort's plan does not depend on the
    // positions, so both are made first.
    if (!p.check && !p.fwd_fused && !profile_now && pbc_mask(s) == 7 && s->nlocal > 0 &&
        s->total_cells > 0 && (s->state == FULL_REBUILD || needs_rebuild_with(s, false))) {
        s->state = FULL_REBUILD;
        TRY(sort_plan(s, &p.sort_due, &p.periodic_sort));
        s->pk_valid = false;
        if (p.sort_due) TRY(counts_zero(s, s->total_cells));
        launch_initial_pbc(s->st, s->nlocal, s->A, s->dt, s->pending_final, p.fused_zero,
                           geom_of(s), s->bvel, grid_of(s), p.sort_due ? s->sort_cell.p : nullptr,
                           s->cell_counts.p);
        s->pending_final = false;
        p.pbc_done = true;
        TRY(check_launch(s));
        timer_end(s, T_INTEGRATE);
        *out = p;
        return SOIL_OK;
    }
    // Forward comm rides on the integration pass when this step keeps its
    // lists unless the displacement check trips (ghost images written from
    // their roots' new positions; a step that rebuilds replaces them).
    FwdArgs fw;
    if (p.fwd_fused) fw = fwd_args(s, p.fused_zero);
    if (s->pending_final)
        launch_final_initial(s->st, s->nlocal, s->A, s->dt, p.fused_zero,
                             p.check ? s->lbx.p : nullptr, s->lby.p, s->lbz.p, s->nlocal,
                             displacement_threshold_sq(s), s->pbc_box, s->dflags, pbc_mask(s),
                             p.fwd_fused ? &fw : nullptr);
    else
        launch_initial(s->st, s->nlocal, s->A, s->dt, p.fused_zero, p.check ? s->lbx.p : nullptr,
                       s->lby.p, s->lbz.p, s->nlocal, displacement_threshold_sq(s), s->pbc_box,
                       s->dflags, pbc_mask(s), p.fwd_fused ? &fw : nullptr);
    s->pending_final = false;
    TRY(check_launch(s));
    timer_end(s, T_INTEGRATE);
    *out = p;
    return SOIL_OK;
}

// The rest of a timestep after its integration pass: decide_rebuild, the
// rebuild phases when due, forward comm, the consumer, reverse comm and the
// final half-kick (applied now when `last`, else deferred into the next
// step's integration pass).
int step_rest(soil_sys* s, const StepPlan& p, bool last) {
    // decide_rebuild
    if (s->state == COMMUNICATE_ONLY) {
        bool disp = false;
        if (p.check) {
            TRY(read_flags(s));
            disp = s->hflags->rebuild != 0;
        }
        if (needs_rebuild_with(s, disp)) s->state = FULL_REBUILD;
        else s->steps_since_build += 1;
    }
    TRY(phase_remove_ghosts(s));
    timer_begin(s, T_ZERO);
    if (!p.fused_zero && (p.nz > 0 || !p.overwrite)) TRY(phase_zero_forces(s));
    timer_end(s, T_ZERO);
    timer_begin(s, T_PBC);
    TRY(phase_shrink_wrap(s));
    // A rebuild step of a fully periodic box wraps its locals and bins them
    // for the sort in one pass: the sort's plan (grid, whether it runs) does
    // not depend on the wrap, so it is made first.
    const bool pbc_cells = p.pbc_done || (s->state == FULL_REBUILD && pbc_mask(s) == 7 &&
                                          s->nlocal > 0 && s->total_cells > 0);
    bool sort_due = p.sort_due, periodic_sort = p.periodic_sort;
    if (p.pbc_done) {
        // wrapped (and binned) in the integration pass
    } else if (pbc_cells) {
        TRY(sort_plan(s, &sort_due, &periodic_sort));
        s->pk_valid = false;
        if (sort_due) {
            TRY(counts_zero(s, s->total_cells));
            launch_pbc_cells(s->st, s->nlocal, s->A, geom_of(s), s->bvel, grid_of(s),
                             s->sort_cell.p, s->cell_counts.p);
        } else {
            launch_pbc(s->st, s->nlocal, s->A, geom_of(s), s->bvel);
        }
        TRY(check_launch(s));
    } else {
        TRY(phase_pbc(s));
    }
    timer_end(s, T_PBC);
    timer_begin(s, T_SORT);
    s->forces_dead = p.overwrite;  // the built-in consumer rewrites every force below
    const int sorted = !pbc_cells ? phase_sort(s)
                     : sort_due   ? sort_run(s, periodic_sort, true)
                                  : SOIL_OK;
    s->forces_dead = false;
    TRY(sorted);
    timer_end(s, T_SORT);
    timer_begin(s, T_BORDERS);
    TRY(phase_borders_defer(s, true));  // read back at the neighbor build's synchronisation
    timer_end(s, T_BORDERS);
    timer_begin(s, T_FORWARD);
    if (s->state == COMMUNICATE_ONLY && !p.fwd_fused) TRY(forward_comm(s, p.fused_zero));
    timer_end(s, T_FORWARD);
    timer_begin(s, T_NEIGHBOR);
    TRY(phase_neighbor(s));
    timer_end(s, T_NEIGHBOR);
    // With newton, the grouped consumer folds ghost forces into their roots
    // in the same kernel (reverse_send_force's fold order); otherwise the
    // force and reverse-comm phases run apart.
    const bool fold_fused = consumer_folds(s);
    timer_begin(s, T_FORCE);
    if (fold_fused) {
        TRY(launch_consumer(s, true));
        s->reverse_gen = s->border_gen;
    } else {
        TRY(phase_force(s));
    }
    timer_end(s, T_FORCE);
    timer_begin(s, T_REVERSE);
    if (!fold_fused && reverse_needed(s)) TRY(phase_reverse_comm(s));
    timer_end(s, T_REVERSE);
    if (last) {
        timer_begin(s, T_FINAL);
        TRY(phase_final(s));
        timer_end(s, T_FINAL);
    } else {
        s->pending_final = true;
        s->steps_done += 1;
    }
    return SOIL_OK;
}

// One full timestep.  Fusions that keep every result bit-identical:
//  - force zeroing folded into initial (locals) and forward comm (ghosts),
//    or dropped when the built-in consumer overwrites every force;
//  - the displacement check folded into the initial integration pass;
//  - final(t) folded into initial(t+1) when nothing touches velocities
//    between them (the streaming profile of the first shear step does);
//  - forward comm folded into the integration pass (fused_forward_ok);
//  - reverse comm folded into the built-in consumer (newton, grouped
//    sequences).
int full_step(soil_sys* s, bool last) {
    StepPlan p;
    TRY(step_integrate(s, &p));
    return step_rest(s, p, last);
}

// ---- device-resident steps -------------------------------------------------

// Steps that may run inside one k_steps launch from the current state: the
// step keeps its lists exactly when its displacement check passes (every = 0
// with the check on), nothing else a step does needs the host (no hook, no
// deform, shear or shrink-wrap, no #[zero] planes, #[reverse] planes only
// with the folding consumer, no phase timers), the built-in consumer (if
// any) runs on grouped sequences, and no periodic sort falls due.  0: none.
uint64_t resident_limit(const soil_sys* s, uint64_t want) {
    const char* env = std::getenv("SOIL_RESIDENT_STEPS");
    const int mode = env ? std::atoi(env) : 2;  // 0 off, 1 always, 2 auto
    if (mode == 0) return 0;
    if (mode == 2 && s->nlocal > kResidentAutoMaxAtoms) return 0;
    if (s->hook || s->timing_mask || !s->check || s->every != 0) return 0;
    if (s->state != COMMUNICATE_ONLY || !displacement_needed(s) || needs_rebuild_with(s, false))
        return 0;
    if (!fused_forward_allowed(s)) return 0;
    const bool consumer = builtin_consumer(s);
    if (consumer && force_variant() != SOIL_FORCE_CSR && !seq_consumer(s)) return 0;
    int idx[kMaxPlanes], nz, nr;
    zero_planes_of(s, SOIL_COL_ZERO, idx, &nz);
    zero_planes_of(s, SOIL_COL_REVERSE, idx, &nr);
    if (nz > 0 || (nr > 0 && !(consumer && s->newton))) return 0;
    uint64_t lim = want;
    if (s->sort_every > 0) {
        if (s->sort_counter + 1 >= s->sort_every) return 0;
        lim = std::min<uint64_t>(lim, s->sort_every - s->sort_counter - 1);
    }
    return lim;
}

// Up to `max` communicate-only steps in one launch; *done of them complete.
// *tripped: the next step's integration pass also ran and its displacement
// check tripped (that step continues on the host from decide_rebuild, with
// *plan).
int resident_steps(soil_sys* s, uint64_t max, uint64_t* done, bool* tripped, StepPlan* plan) {
    const StepPlan p = plan_step(s);
    const bool consumer = builtin_consumer(s);
    if (consumer && force_variant() != SOIL_FORCE_GATHER) TRY(pk_ready(s));
    StepsArgs a;
    std::memset(&a, 0, sizeof(a));
    a.c = s->A;
    a.nlocal = s->nlocal;
    a.dt = s->dt;
    a.zero_force = p.fused_zero ? 1 : 0;
    a.first_fused = s->pending_final ? 1 : 0;
    a.ck = make_check(s->lbx.p, s->lby.p, s->lbz.p, s->nlocal, displacement_threshold_sq(s),
                      s->pbc_box, s->dflags, pbc_mask(s));
    a.fw = fwd_args(s, p.fused_zero);
    a.walk = 0;
    int kind = 0;
    if (consumer) {
        if (!s->in_lists_valid) TRY(build_in_lists(s));
        kind = s->newton ? 2 : 1;
        const int v = force_variant();
        if (v == SOIL_FORCE_CSR) {
            TRY(csr_with_order(s, &a.fc));
            zero_planes_of(s, SOIL_COL_REVERSE, a.fa.rev.idx, &a.fa.rev.n);
            a.walk = 2;
        } else {
            if (!s->seq_valid) TRY(build_seq(s));
            a.fa = consumer_args(s);
            a.walk = (v == SOIL_FORCE_TILES4 || v == SOIL_FORCE_TILES2) ? 0 : 1;
        }
    }
    a.max_steps = max;
    TRY(ensure(s, s->rstate, 8));
    a.bar = reinterpret_cast<GridBar*>(s->rstate.p);
    a.out = s->rstate.p + 2;
    a.trip = s->rstate.p + 4;
    a.flags = s->dflags;
    int grid = 0;
    const bool pk = a.walk == 2 ? a.fc.pk != nullptr : a.fa.q.pk != nullptr;
    if (steps_grid(kind, a.walk, pk, s->nlocal, &grid))
        return fail(s->ctx, SOIL_ERR_CUDA, "no cooperative occupancy for the resident steps");
    CK(cudaMemsetAsync(s->rstate.p, 0, 8 * 4, s->st));
    CK(cudaMemsetAsync(&s->dflags->rebuild, 0, 4, s->st));
    CK(cudaMemsetAsync(&s->dflags->error, 0, 4, s->st));
    CK(launch_steps(s->st, a, kind, a.walk, pk, grid));
    CK(cudaMemcpyAsync(s->hword, a.out, 8, cudaMemcpyDeviceToHost, s->st));
    TRY(read_flags(s));
    if (s->hflags->error & SOIL_STEPS_ERR_BARRIER)
        return fail(s->ctx, SOIL_ERR_CUDA, "resident steps: a grid barrier wait ran out");
    *done = s->hword[0];
    *tripped = s->hword[1] != 0;
    if (*done > max || (!*tripped && *done != max))
        return fail(s->ctx, SOIL_ERR_CUDA, "resident steps: inconsistent step count");
    s->steps_done += *done;
    s->steps_since_build += *done;
    if (s->sort_every > 0) s->sort_counter += *done;
    // every completed step leaves its final half-kick pending; a tripped
    // step's integration pass applied the last one
    s->pending_final = !*tripped;
    *plan = p;
    plan->check = true;
    plan->fwd_fused = true;
    return SOIL_OK;
}

// soil_step: communicate-only stretches run resident when resident_limit
// allows (at least two steps), every other step through full_step.
int step_many(soil_sys* s, uint64_t n) {
    if (s->view_out) s->pk_valid = false;  // a view's holder may have moved atoms
    uint64_t k = 0;
    while (k < n) {
        const uint64_t lim = resident_limit(s, n - k);
        if (lim >= 2) {
            uint64_t done = 0;
            bool tripped = false;
            StepPlan p;
            TRY(resident_steps(s, lim, &done, &tripped, &p));
            k += done;
            if (tripped) {  // step k + 1: integrated, its check tripped
                TRY(step_rest(s, p, k + 1 == n));
                k += 1;
            } else if (k == n) {  // the call ends on a resident step
                launch_final(s->st, s->nlocal, s->A, s->dt);
                s->pending_final = false;
                TRY(check_launch(s));
            }
            continue;
        }
        TRY(full_step(s, k + 1 == n));
        k += 1;
    }
    return SOIL_OK;
}

}  // namespace soil_host

using namespace soil_host;

namespace soil {
// Records `msg` as the context's last error (ctx may be NULL) and returns status.
int set_ctx_error(soil_ctx* ctx, int status, const char* msg) {
    if (ctx) {
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->err = msg;
    }
    return status;
}
}  // namespace soil

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int soil_abi_version(void) { return SOIL_ABI_VERSION; }

int soil_ctx_create(int device, uint64_t hbm_budget_bytes, soil_ctx** out) {
    if (!out) return SOIL_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) {
        cudaGetLastError();
        return SOIL_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return SOIL_ERR_NO_DEVICE;
    }
    soil_ctx* c = new (std::nothrow) soil_ctx();
    if (!c) return SOIL_ERR_OOM;
    c->device = device;
    c->budget = hbm_budget_bytes;
    // Device arrays come from a stream-ordered pool of this context that keeps
    // freed memory (the budget counts what is in use); growth of a system's
    // arrays then neither synchronises the device nor maps new memory.
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return SOIL_ERR_CUDA;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    *out = c;
    return SOIL_OK;
}

int soil_ctx_destroy(soil_ctx* ctx) {
    // the pool's memory goes back once the last outstanding free has run
    if (ctx && ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return SOIL_OK;
}

const char* soil_last_error(const soil_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int soil_ctx_bytes_in_use(const soil_ctx* ctx, uint64_t* out) {
    if (!ctx || !out) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    *out = ctx->in_use;
    return SOIL_OK;
}

int soil_ctx_alloc_count(const soil_ctx* ctx, uint64_t* allocs, uint64_t* frees) {
    if (!ctx) return SOIL_ERR_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (allocs) *allocs = ctx->allocs;
    if (frees) *frees = ctx->frees;
    return SOIL_OK;
}

int soil_sys_create(soil_ctx* ctx, const soil_box* box, const soil_neigh_cfg* cfg, double dt,
                    soil_sys** out) {
    if (!ctx || !box || !cfg || !out) return SOIL_ERR_INVALID;
    *out = nullptr;
    for (int d = 0; d < 3; ++d)
        if (!(box->hi[d] > box->lo[d]))
            return fail(ctx, SOIL_ERR_INVALID, "box axis %d has hi <= lo", d);
    if (!(cfg->skin_fraction >= 1.0) || !(cfg->bin_size > 0.0) || cfg->additive_skin < 0.0 ||
        (cfg->filter != SOIL_FILTER_FP64 && cfg->filter != SOIL_FILTER_FP32_RECHECK))
        return fail(ctx, SOIL_ERR_INVALID, "invalid neighbor config");
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, SOIL_ERR_NO_DEVICE, "cudaSetDevice(%d) failed", ctx->device);
    }
    soil_sys* s = new (std::nothrow) soil_sys();
    if (!s) return SOIL_ERR_OOM;
    s->ctx = ctx;
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return fail(ctx, SOIL_ERR_CUDA, "cudaStreamCreate failed");
    }
    // decompose_domain on a 1x1x1 grid (domain.rs:235-296)
    for (int d = 0; d < 3; ++d) {
        s->blo[d] = box->lo[d];
        s->bhi[d] = box->hi[d];
        s->size[d] = box->hi[d] - box->lo[d];
        const double delta = s->size[d] / 1.0;
        s->sub_lo[d] = box->lo[d] + delta * 0.0;
        s->sub_hi[d] = box->lo[d] + delta * 1.0;
        s->sub_len[d] = delta;
    }
    s->dt = dt;
    s->skin_fraction = cfg->skin_fraction;
    s->bin_min_size = cfg->bin_size;
    s->every = cfg->every;
    s->sort_every = cfg->sort_every;
    s->check = cfg->check != 0;
    s->newton = cfg->newton != 0;
    s->additive_skin = cfg->additive_skin;
    s->filter = cfg->filter;
    int r;
    if ((r = dev_alloc(s, (void**)&s->dflags, sizeof(DevFlags))) != SOIL_OK ||
        cudaHostAlloc((void**)&s->hflags, sizeof(DevFlags), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc((void**)&s->hword, 2 * kBorderStateWords * 4, cudaHostAllocMapped) !=
            cudaSuccess ||
        cudaHostGetDevicePointer((void**)&s->hflags_dev, s->hflags, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&s->hword_dev, s->hword, 0) != cudaSuccess) {
        cudaGetLastError();
        soil_sys_destroy(s);
        return r != SOIL_OK ? r : fail(ctx, SOIL_ERR_OOM, "pinned allocation failed");
    }
    cudaMemsetAsync(s->dflags, 0, sizeof(DevFlags), s->st);
    *out = s;
    return SOIL_OK;
}

int soil_sys_destroy(soil_sys* s) {
    if (!s) return SOIL_OK;
    if (s->batch) soil_batch_remove(s->batch, s);
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->A.x) free_cols(s, s->A);
    if (s->B.x) free_cols(s, s->B);
    auto fr = [&](auto& a) {
        dev_free(s, a.p, a.cap * sizeof(*a.p));
        a.p = nullptr;
        a.cap = 0;
    };
    fr(s->lbx); fr(s->lby); fr(s->lbz);
    fr(s->sort_cell); fr(s->sort_perm); fr(s->sorted_local_cell); fr(s->sort_start); fr(s->ghost_tmp);
    fr(s->cell_counts); fr(s->cell_start); fr(s->cell_cursor);
    fr(s->atom_cell); fr(s->sorted_atoms); fr(s->asi); fr(s->rowcount); fr(s->offsets); fr(s->indices);
    fr(s->row_slots); fr(s->sp); fr(s->spf);
    fr(s->sel_flag); fr(s->sel_pos); fr(s->sel_out); fr(s->sel_cnt); fr(s->ext);
    fr(s->fold_roots); fr(s->fold_nroots);
    for (int k = 0; k < 2; ++k) { fr(s->slot_tag[k]); fr(s->slot_val[k]); }
    fr(s->in_count); fr(s->in_start); fr(s->in_cursor); fr(s->in_list); fr(s->in_split);
    fr(s->seq_cnt); fr(s->grp_cnt); fr(s->grp_start); fr(s->seq); fr(s->seq_owner);
    fr(s->rstate); fr(s->scan1p); fr(s->root_order); fr(s->pk);
    fr(s->ghost_root); fr(s->ghost_chain);
    fr(s->fold_start); fr(s->fold_list);
    for (auto& a : s->send) fr(a);
    fr(s->bstate);
    fr(s->bcount); fr(s->boff);
    fr(s->face_flags);
    fr(s->scan_tmp); fr(s->d_stencil); fr(s->stage); fr(s->d_colptrs);
    resolve_timers(s);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    if (s->ev_counts) cudaEventDestroy(s->ev_counts);
    if (s->dflags) dev_free(s, s->dflags, sizeof(DevFlags));
    if (s->hflags) cudaFreeHost(s->hflags);
    if (s->hword) cudaFreeHost(s->hword);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return SOIL_OK;
}

int soil_sys_register_column(soil_sys* s, const char* name, int32_t width, uint32_t flags,
                             int32_t* col_out) {
    if (!s || !name || width <= 0) return SOIL_ERR_INVALID;
    if (s->setup_done || s->nlocal > 0)
        return fail(s->ctx, SOIL_ERR_STATE, "columns must be registered before atoms are added");
    for (const ColMeta& c : s->cols)
        if (c.name == name)
            return fail(s->ctx, SOIL_ERR_INVALID, "AtomData column '%s' already registered", name);
    if ((int)s->cols.size() >= kMaxCols || s->nplanes + width > kMaxPlanes)
        return fail(s->ctx, SOIL_ERR_CAPACITY, "at most %d columns / %d f64 planes", kMaxCols,
                    kMaxPlanes);
    s->cols.push_back({name, (int)width, flags, s->nplanes});
    s->nplanes += width;
    if (col_out) *col_out = (int32_t)s->cols.size() - 1;
    return SOIL_OK;
}

int soil_sys_add_atoms(soil_sys* s, uint64_t n, const uint32_t* tag, const uint32_t* type,
                       const double* pos3, const double* vel3, const double* mass,
                       const double* cutoff_radius, const double* const* columns) {
    if (!s || (n && (!tag || !pos3 || !vel3 || !mass || !cutoff_radius))) return SOIL_ERR_INVALID;
    if (s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "atoms must be added before setup");
    // one host pass: validation and the cutoff radii's extremes
    double cmin = s->cut_min_local, cmax = s->cut_max_local;
    for (uint64_t i = 0; i < n; ++i) {
        if (!(mass[i] > 0.0) || !(cutoff_radius[i] >= 0.0))
            return fail(s->ctx, SOIL_ERR_INVALID, "atom %llu: mass must be > 0 and cutoff >= 0",
                        (unsigned long long)i);
        cmin = std::fmin(cmin, cutoff_radius[i]);
        cmax = std::fmax(cmax, cutoff_radius[i]);
    }
    const uint64_t base = s->nlocal;
    TRY(grow_atoms(s, base + n, base));
    if (n == 0) return SOIL_OK;
    // staging: positions and velocities, then the widest column, side by side
    uint64_t wmax = 0;
    for (const ColMeta& m : s->cols) wmax = std::max<uint64_t>(wmax, (uint64_t)m.width);
    TRY(ensure(s, s->stage, 6 * n + wmax * n));
    double* st3 = s->stage.p;
    double* sv3 = s->stage.p + 3 * n;
    double* scol = s->stage.p + 6 * n;
    CK(cudaMemcpyAsync(st3, pos3, n * 24, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(sv3, vel3, n * 24, cudaMemcpyHostToDevice, s->st));
    launch_deinterleave3(s->st, n, st3, s->A.x + base, s->A.y + base, s->A.z + base);
    launch_deinterleave3(s->st, n, sv3, s->A.vx + base, s->A.vy + base, s->A.vz + base);
    CK(cudaMemsetAsync(s->A.fx + base, 0, n * 8, s->st));
    CK(cudaMemsetAsync(s->A.fy + base, 0, n * 8, s->st));
    CK(cudaMemsetAsync(s->A.fz + base, 0, n * 8, s->st));
    CK(cudaMemcpyAsync(s->A.mass + base, mass, n * 8, cudaMemcpyHostToDevice, s->st));
    launch_inverse(s->st, n, s->A.mass + base, s->A.inv_mass + base);
    CK(cudaMemcpyAsync(s->A.cut + base, cutoff_radius, n * 8, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->A.tag + base, tag, n * 4, cudaMemcpyHostToDevice, s->st));
    if (type) CK(cudaMemcpyAsync(s->A.type + base, type, n * 4, cudaMemcpyHostToDevice, s->st));
    else CK(cudaMemsetAsync(s->A.type + base, 0, n * 4, s->st));
    for (int d = 0; d < 3; ++d) CK(cudaMemsetAsync(s->A.img + d * s->acap + base, 0, n * 4, s->st));
    CK(cudaMemsetAsync(s->A.origin + base, 0, n * 4, s->st));
    bool col_pending = false;
    for (size_t c = 0; c < s->cols.size(); ++c) {
        const ColMeta& m = s->cols[c];
        if (columns && columns[c]) {
            if (col_pending) CK(cudaStreamSynchronize(s->st));  // scol is reused
            CK(cudaMemcpyAsync(scol, columns[c], (uint64_t)m.width * n * 8,
                               cudaMemcpyHostToDevice, s->st));
            launch_deinterleave_w(s->st, n, m.width, scol, s->A.planes[m.plane0] + base, s->acap);
            col_pending = true;
        } else {
            for (int w = 0; w < m.width; ++w)
                CK(cudaMemsetAsync(s->A.planes[m.plane0 + w] + base, 0, n * 8, s->st));
        }
    }
    TRY(check_launch(s));
    TRY(sync(s));
    s->cut_min_local = cmin;
    s->cut_max_local = cmax;
    s->nlocal += n;
    return SOIL_OK;
}

int soil_sys_setup(soil_sys* s) {
    if (!s) return SOIL_ERR_INVALID;
    if (s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "setup already done");
    TRY(grow_atoms(s, s->nlocal + 1, s->nlocal));
    // comm_setup (comm.rs:253-283): rank 0 of 1x1x1, every axis periodic; the
    // shifts are applied in phase_borders.
    // neighbor_setup (neighbor.rs:604-665), comm size 1
    double max_skin = 0.0;
    if (s->nlocal) max_skin = std::fmax(0.0, s->cut_max_local);
    const double max_cutoff = max_skin > 0.0 ? 2.0 * max_skin * s->skin_fraction : s->bin_min_size;
    const double min_skin = s->nlocal ? s->cut_min_local : DBL_MAX;
    double buffer = 0.0;
    if (min_skin < DBL_MAX * 0.5) {
        buffer = (s->skin_fraction - 1.0) * min_skin;
        if (s->additive_skin != 0.0) buffer = buffer + 0.5 * s->additive_skin;
    }
    const double ghost_cut = std::fmax(max_cutoff + 2.0 * buffer, s->domain_ghost_cutoff);
    s->ghost_cutoff = ghost_cut;
    s->cached_max_cutoff = max_cutoff;
    s->domain_ghost_cutoff = ghost_cut;
    if (s->bin_min_size < max_cutoff) s->bin_min_size = max_cutoff;
    compute_bin_grid(s);
    if (s->total_cells >= 0x7fffffffull)
        return fail(s->ctx, SOIL_ERR_CAPACITY, "bin grid of %llu cells is too large",
                    (unsigned long long)s->total_cells);
    if (s->shear && (pbc_mask(s) & 3) != 3)
        return fail(s->ctx, SOIL_ERR_INVALID,
                    "Lees-Edwards shear needs periodic x and y (setup_deform, lib.rs:365-371)");
    // setup_deform (soil_deform/src/lib.rs:346-420)
    for (int d = 0; d < 3; ++d)
        if (s->axis[d].style) {
            s->axis[d].lo0 = s->blo[d];
            s->axis[d].hi0 = s->bhi[d];
        }
    s->shear_initialized = false;
    s->deform_initialized = true;
    s->deform_step = 0;
    s->setup_done = true;
    TRY(update_colptrs(s));
    return SOIL_OK;
}

int soil_sys_set_shear(soil_sys* s, double erate) {
    if (!s) return SOIL_ERR_INVALID;
    if (s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "set the shear rate before setup");
    s->shear = true;
    s->shear_rate = erate;
    return SOIL_OK;
}

int soil_sys_set_deform(soil_sys* s, int32_t dim, int32_t style, double a, double b,
                        uint64_t stage_steps) {
    if (!s) return SOIL_ERR_INVALID;
    if (dim < 0 || dim > 2 || style < SOIL_DEFORM_NONE || style > SOIL_DEFORM_FINAL)
        return fail(s->ctx, SOIL_ERR_INVALID, "deform: dim in 0..2, style SOIL_DEFORM_*");
    if (s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "set deform styles before setup");
    soil_sys::AxisDeform& ax = s->axis[dim];
    ax.style = style;
    ax.a = a;
    ax.b = b;
    ax.stage_steps = stage_steps;
    return SOIL_OK;
}

int soil_sys_set_deform_remap(soil_sys* s, int32_t remap) {
    if (!s) return SOIL_ERR_INVALID;
    s->remap = remap != 0;
    return SOIL_OK;
}

int soil_sys_get_box(soil_sys* s, double* lo, double* hi, double* tilt) {
    if (!s || !lo || !hi || !tilt) return SOIL_ERR_INVALID;
    for (int d = 0; d < 3; ++d) {
        lo[d] = s->blo[d];
        hi[d] = s->bhi[d];
        tilt[d] = s->tilt[d];
    }
    return SOIL_OK;
}

int soil_sys_set_harmonic(soil_sys* s, double k, int32_t radius_col) {
    if (!s) return SOIL_ERR_INVALID;
    if (k != 0.0 && (radius_col < 0 || (size_t)radius_col >= s->cols.size() ||
                     s->cols[radius_col].width != 1))
        return fail(s->ctx, SOIL_ERR_INVALID, "radius column must be a registered width-1 column");
    if (s->batch) return fail(s->ctx, SOIL_ERR_STATE, "the force of a batched system is fixed");
    s->harmonic_k = k;
    s->radius_col = radius_col;
    s->pk_valid = false;
    s->in_lists_valid = false;
    s->seq_valid = false;
    s->order_valid = false;
    return SOIL_OK;
}

int soil_sys_set_force_hook(soil_sys* s, soil_force_fn fn, void* user) {
    if (!s) return SOIL_ERR_INVALID;
    if (s->batch) return fail(s->ctx, SOIL_ERR_STATE, "the force of a batched system is fixed");
    s->hook = fn;
    s->hook_user = user;
    return SOIL_OK;
}

int soil_step(soil_sys* s, uint64_t nsteps) {
    if (!s) return SOIL_ERR_INVALID;
    if (!s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "soil_sys_setup has not run");
    if (s->batch) return fail(s->ctx, SOIL_ERR_STATE, "a batched system steps through its batch");
    return step_many(s, nsteps);
}

int soil_sys_sync(soil_sys* s) {
    if (!s) return SOIL_ERR_INVALID;
    return sync(s);
}

int soil_sys_stream(soil_sys* s, void** out) {
    if (!s || !out) return SOIL_ERR_INVALID;
    *out = (void*)s->st;
    return SOIL_OK;
}

#define PHASE_ENTRY(name)                                                                  \
    int soil_phase_##name(soil_sys* s) {                                                   \
        if (!s) return SOIL_ERR_INVALID;                                                   \
        if (!s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "soil_sys_setup has not run"); \
        if (s->pending_final) {                                                            \
            launch_final(s->st, s->nlocal, s->A, s->dt);                                   \
            s->pending_final = false;                                                      \
        }                                                                                  \
        return phase_##name(s);                                                            \
    }
PHASE_ENTRY(deform)
PHASE_ENTRY(initial)
PHASE_ENTRY(decide_rebuild)
PHASE_ENTRY(remove_ghosts)
PHASE_ENTRY(zero_forces)
PHASE_ENTRY(shrink_wrap)
PHASE_ENTRY(pbc)
PHASE_ENTRY(sort)
PHASE_ENTRY(borders)
PHASE_ENTRY(forward_comm)
PHASE_ENTRY(neighbor)
PHASE_ENTRY(force)
PHASE_ENTRY(reverse_comm)
PHASE_ENTRY(final)

int soil_sys_counts(soil_sys* s, soil_counts* o) {
    if (!s || !o) return SOIL_ERR_INVALID;
    std::memset(o, 0, sizeof(*o));
    o->nlocal = s->nlocal;
    o->nghost = s->nghost;
    o->npairs = s->npairs;
    o->step = s->steps_done;
    o->rebuilds = s->rebuilds;
    o->sorts = s->sorts;
    o->steps_since_build = s->steps_since_build;
    o->filter_candidates = s->hflags ? s->hflags->candidates : 0;
    o->filter_rechecked = s->hflags ? s->hflags->rechecked : 0;
    o->comm_state = s->state;
    o->triclinic = s->triclinic ? 1 : 0;
    for (int d = 0; d < 3; ++d) o->bin_count[d] = s->bin_count[d];
    o->nstencil_forward = (int32_t)s->stencil_fwd.size();
    o->ghost_cutoff = s->ghost_cutoff;
    o->max_cutoff = s->cached_max_cutoff;
    o->tilt_xy = s->tilt[0];
    return SOIL_OK;
}

static int flush_pending(soil_sys* s) {
    if (s->pending_final) {
        launch_final(s->st, s->nlocal, s->A, s->dt);
        s->pending_final = false;
    }
    return check_launch(s);
}

int soil_sys_get_atoms(soil_sys* s, uint64_t first, uint64_t n, uint32_t* tag, double* pos3,
                       double* vel3, double* force3, int32_t* image3, int32_t* origin_index) {
    if (!s) return SOIL_ERR_INVALID;
    if (first + n > s->nlocal + s->nghost) return fail(s->ctx, SOIL_ERR_INVALID, "range out of bounds");
    if (n == 0) return SOIL_OK;
    TRY(flush_pending(s));
    TRY(ensure(s, s->stage, 3 * n));
    const uint64_t f = first;
    auto get3 = [&](double* dst, double* a, double* b, double* c) -> int {
        if (!dst) return SOIL_OK;
        launch_interleave3(s->st, n, s->stage.p, a + f, b + f, c + f);
        CK(cudaMemcpyAsync(dst, s->stage.p, n * 24, cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        return SOIL_OK;
    };
    TRY(get3(pos3, s->A.x, s->A.y, s->A.z));
    TRY(get3(vel3, s->A.vx, s->A.vy, s->A.vz));
    TRY(get3(force3, s->A.fx, s->A.fy, s->A.fz));
    if (tag) CK(cudaMemcpyAsync(tag, s->A.tag + f, n * 4, cudaMemcpyDeviceToHost, s->st));
    if (origin_index) CK(cudaMemcpyAsync(origin_index, s->A.origin + f, n * 4, cudaMemcpyDeviceToHost, s->st));
    if (image3) {
        int32_t* st3 = (int32_t*)s->stage.p;
        launch_interleave3i(s->st, n, st3, s->A.img + f, s->A.img + s->acap + f,
                            s->A.img + 2 * s->acap + f);
        CK(cudaMemcpyAsync(image3, st3, n * 12, cudaMemcpyDeviceToHost, s->st));
    }
    TRY(check_launch(s));
    return sync(s);
}

int soil_sys_get_column(soil_sys* s, int32_t col, uint64_t first, uint64_t n, double* out) {
    if (!s || !out || col < 0 || (size_t)col >= s->cols.size()) return SOIL_ERR_INVALID;
    if (first + n > s->nlocal + s->nghost) return fail(s->ctx, SOIL_ERR_INVALID, "range out of bounds");
    if (n == 0) return SOIL_OK;
    TRY(flush_pending(s));
    const ColMeta& m = s->cols[col];
    TRY(ensure(s, s->stage, (uint64_t)m.width * n));
    launch_interleave_w(s->st, n, m.width, s->stage.p, s->A.planes[m.plane0] + first, s->acap);
    CK(cudaMemcpyAsync(out, s->stage.p, (uint64_t)m.width * n * 8, cudaMemcpyDeviceToHost, s->st));
    TRY(check_launch(s));
    return sync(s);
}

int soil_sys_get_neighbor(soil_sys* s, uint32_t* offsets, uint32_t* indices) {
    if (!s) return SOIL_ERR_INVALID;
    if (s->rebuilds == 0) return fail(s->ctx, SOIL_ERR_STATE, "no neighbor list built yet");
    if (offsets) CK(cudaMemcpyAsync(offsets, s->offsets.p, (s->nlocal + 1) * 4, cudaMemcpyDeviceToHost, s->st));
    if (indices && s->npairs)
        CK(cudaMemcpyAsync(indices, s->indices.p, s->npairs * 4, cudaMemcpyDeviceToHost, s->st));
    return sync(s);
}

int soil_sys_num_swaps(soil_sys* s, int32_t* out) {
    if (!s || !out) return SOIL_ERR_INVALID;
    *out = s->nswaps;
    return SOIL_OK;
}

int soil_sys_get_swap(soil_sys* s, int32_t k, uint64_t* recv_start, uint64_t* recv_count,
                      double periodic_offset[3], double vel_offset[3], uint32_t* send_indices) {
    if (!s || k < 0 || k >= s->nswaps) return SOIL_ERR_INVALID;
    const SwapHost& h = s->swaps[k];
    if (recv_start) *recv_start = h.recv_start;
    if (recv_count) *recv_count = h.recv_count;
    for (int d = 0; d < 3; ++d) {
        if (periodic_offset) periodic_offset[d] = h.off[d];
        if (vel_offset) vel_offset[d] = h.voff[d];
    }
    if (send_indices && h.send_count)
        CK(cudaMemcpyAsync(send_indices, s->send[k].p, h.send_count * 4, cudaMemcpyDeviceToHost, s->st));
    return sync(s);
}

int soil_sys_get_swap_sends(soil_sys* s, int32_t k, uint64_t* count) {
    if (!s || !count || k < 0 || k >= s->nswaps) return SOIL_ERR_INVALID;
    *count = s->swaps[k].send_count;
    return SOIL_OK;
}

int soil_sys_set_boundary(soil_sys* s, const int32_t* type, double shrink_padding) {
    if (!s || !type) return SOIL_ERR_INVALID;
    for (int d = 0; d < 3; ++d)
        if (type[d] < SOIL_BOUNDARY_PERIODIC || type[d] > SOIL_BOUNDARY_SHRINK)
            return fail(s->ctx, SOIL_ERR_INVALID, "boundary type of axis %d: SOIL_BOUNDARY_*", d);
    if (s->setup_done) return fail(s->ctx, SOIL_ERR_STATE, "set boundaries before setup");
    for (int d = 0; d < 3; ++d) s->btype[d] = type[d];
    s->shrink_padding = shrink_padding;
    return SOIL_OK;
}

int soil_sys_get_sort_perm(soil_sys* s, uint32_t* perm) {
    if (!s || !perm) return SOIL_ERR_INVALID;
    if (!s->perm_valid) return fail(s->ctx, SOIL_ERR_STATE, "no spatial sort has run");
    CK(cudaMemcpyAsync(perm, s->sort_perm.p, s->nlocal * 4, cudaMemcpyDeviceToHost, s->st));
    return sync(s);
}

int soil_sys_enable_slots(soil_sys* s, uint32_t max_contacts, uint32_t width) {
    if (!s) return SOIL_ERR_INVALID;
    if (max_contacts == 0 || max_contacts > 1024 || width == 0 || width > 64)
        return fail(s->ctx, SOIL_ERR_INVALID, "slots: max_contacts in [1, 1024], width in [1, 64]");
    if (s->batch) return fail(s->ctx, SOIL_ERR_STATE, "slots are not available to a batched system");
    if (s->slot_max) return fail(s->ctx, SOIL_ERR_STATE, "slots are already enabled");
    s->slot_max = max_contacts;
    s->slot_width = width;
    s->slot_old = 0;
    if (s->acap) {  // otherwise the arrays come with the first capacity (setup)
        const int st = slots_grow(s, s->acap, 0);
        if (st != SOIL_OK) {
            for (int k = 0; k < 2; ++k) {
                dev_free(s, s->slot_tag[k].p, s->slot_tag[k].cap * 4);
                dev_free(s, s->slot_val[k].p, s->slot_val[k].cap * 8);
                s->slot_tag[k] = {};
                s->slot_val[k] = {};
            }
            s->slot_max = s->slot_width = 0;
            return st;
        }
    }
    return SOIL_OK;
}

int soil_sys_get_slots(soil_sys* s, uint32_t* partner_tag, double* payload) {
    if (!s || !partner_tag || !payload) return SOIL_ERR_INVALID;
    if (!s->slot_max) return fail(s->ctx, SOIL_ERR_STATE, "slots are not enabled");
    const uint64_t nt = s->nlocal * s->slot_max;
    const int o = s->slot_old;
    if (nt) {
        CK(cudaMemcpyAsync(partner_tag, s->slot_tag[o].p, nt * 4, cudaMemcpyDeviceToHost, s->st));
        CK(cudaMemcpyAsync(payload, s->slot_val[o].p, nt * s->slot_width * 8,
                           cudaMemcpyDeviceToHost, s->st));
    }
    return sync(s);
}

int soil_sys_view(soil_sys* s, soil_dev_view* out) {
    if (!s || !out) return SOIL_ERR_INVALID;
    TRY(flush_pending(s));
    TRY(make_view(s, out));
    s->view_out = true;  // columns may change between steps until the next rebuild
    return sync(s);  // stream-ordered allocations are ready for every stream
}

uint64_t soil_kernel_launches(void) { return launches_so_far(); }

const char* soil_consumer_kernel(void) {
    switch (soil::force_variant()) {
        case soil::SOIL_FORCE_GATHER: return "k_harmonic";
        case soil::SOIL_FORCE_CSR: return "k_force_csr";
        case soil::SOIL_FORCE_WALK: return "k_force_walk";
        default: return "k_force_seq";
    }
}

int soil_sys_set_timing(soil_sys* s, uint32_t mask) {
    if (!s) return SOIL_ERR_INVALID;
    TRY(sync(s));
    resolve_timers(s);
    s->timing_mask = mask;
    for (int t = 0; t < SOIL_NUM_TIMERS; ++t) {
        s->timer_ms[t] = 0.0;
        s->timer_launches[t] = 0;
        s->timer_intervals[t] = 0;
    }
    return SOIL_OK;
}

int soil_sys_get_timing(soil_sys* s, double* ms, uint64_t* launches, uint64_t* intervals) {
    if (!s) return SOIL_ERR_INVALID;
    TRY(sync(s));
    resolve_timers(s);
    for (int t = 0; t < SOIL_NUM_TIMERS; ++t) {
        if (ms) ms[t] = s->timer_ms[t];
        if (launches) launches[t] = s->timer_launches[t];
        if (intervals) intervals[t] = s->timer_intervals[t];
    }
    return SOIL_OK;
}

const char* soil_timer_name(int32_t i) {
    return (i >= 0 && i < SOIL_NUM_TIMERS) ? kTimerNames[i] : "";
}

}  // extern "C"
