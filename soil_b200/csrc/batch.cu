// batch.cu — the batched engine: many independent systems ("boxes") advanced
// together, every phase one kernel launch over all the boxes that take part.
//
// Each box keeps its own soil_sys state and device arrays.  The batch holds
// the device tables of the boxes' pointers (BoxDev) and per-step values
// (BoxStep), one flags / border-state / pair-total row per box, and the
// segment tables (Span) of every launch.  A step runs, for every box, exactly
// the phase sequence and per-atom arithmetic of soil_step (the host decisions
// are the same functions), so a box's results are bit-identical alone and in
// a batch.  The host waits for the device at most three times per step: for
// the displacement answers after the integration, for the ghost counts after
// the border passes and for the CSR sizes after the pair-count pass; a step
// in which no box rebuilds waits once (or not at all when no box checks).
//
// Host→device traffic goes through per-stage pinned buffers guarded by an
// event, so a buffer is rewritten only after its previous copy finished.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>

#include "batch.cuh"
#include "host_pool.h"
#include "sys_internal.cuh"

using namespace soil;
using namespace soil_host;

#define BCK(call)                                                                               \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail(b->ctx, SOIL_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                    \
    } while (0)

namespace {

// One launch's segment table under construction.
struct SpanBuild {
    std::vector<uint32_t> box, base;
    std::vector<uint64_t> start{0};
    std::vector<uint8_t> flag;
    void clear() {
        box.clear();
        base.clear();
        flag.clear();
        start.assign(1, 0);
    }
    // n elements of box `bx` starting at element `first` of the box
    void add(uint32_t bx, uint64_t n, uint64_t first, uint8_t f = 0) {
        box.push_back(bx);
        base.push_back((uint32_t)first);
        flag.push_back(f);
        start.push_back(start.back() + n);
    }
    // like add, but leaves out empty ranges (element spans only)
    void add_nz(uint32_t bx, uint64_t n, uint64_t first, uint8_t f = 0) {
        if (n) add(bx, n, first, f);
    }
};

// Pinned staging + device region of one stage of a step.
struct Stage {
    uint8_t* h = nullptr;
    uint8_t* d = nullptr;
    size_t cap = 0, used = 0;
    cudaEvent_t ev = nullptr;
    bool pending = false;
    std::deque<SpanBuild> spans;
    size_t nspans = 0;
    std::vector<Span> out;
};

}  // namespace

struct soil_batch {
    soil_ctx* ctx = nullptr;
    cudaStream_t st = nullptr;
    std::vector<soil_sys*> slot;      // nullptr: free slot
    std::vector<cudaStream_t> saved;  // each member's own stream while it is batched
    std::vector<uint32_t> members;    // occupied slots, largest box first
    uint32_t cap = 0;
    std::vector<BoxDev> h_dev;
    std::vector<BoxStep> h_step;
    std::vector<uint8_t> dev_dirty, step_dirty;
    std::vector<std::array<BorderDim, 3>> bds;
    BoxDev* d_dev = nullptr;
    BoxStep* d_step = nullptr;
    DevFlags* d_flags = nullptr;
    DevFlags* h_flags = nullptr;  // pinned
    uint32_t* d_bstate = nullptr;
    uint32_t* h_bread = nullptr;  // pinned
    std::vector<uint32_t> binit;
    uint32_t* d_totals = nullptr;
    uint32_t* h_totals = nullptr;  // pinned
    uint64_t dev_bytes = 0;
    Stage stage[6];
    uint64_t steps = 0, waits = 0, border_retries = 0;
    // stage timers: device time between events recorded around each stage
    struct Timed {
        int stage;
        cudaEvent_t a, z;
    };
    bool timing = false;
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> ev_pool;
    double stage_ms[SOIL_BATCH_NUM_TIMERS] = {};
    uint64_t stage_n[SOIL_BATCH_NUM_TIMERS] = {};
    cudaEvent_t open_a = nullptr;
    cudaEvent_t step_a = nullptr;
    // host time per planning section, waits excluded (and summed apart)
    std::chrono::steady_clock::time_point hlast;
    double host_ms[SOIL_BATCH_NUM_HOST_TIMERS] = {};
    double wait_pending_ms = 0.0;
    std::unique_ptr<HostPool> pool;  // per-box planning threads
    size_t min_parallel = 64;        // fewer boxes are planned on the calling thread
    // per-step scratch
    std::vector<uint8_t> check, full_at_pbc, run, periodic, apply, rebuild, planned;
    // Per-slot copies of the counts the step's serial loops read, so that they
    // do not walk every member's system record (written by the planning
    // threads) on the calling thread.  nlocal and newton are fixed while a
    // system is batched; nghost and cells are refreshed where they change.
    struct Hot {
        uint64_t nlocal = 0, nghost = 0, cells = 0;
        uint8_t newton = 0, cells_valid = 0;
    };
    std::vector<Hot> hot;
};

namespace {

enum { G_INTEGRATE, G_SORT, G_SORT_APPLY, G_BORDERS, G_NEIGHBOR, G_FORCE };

int balloc(soil_batch* b, void** p, uint64_t bytes) {
    if (bytes == 0) bytes = 16;
    TRY(ctx_reserve(b->ctx, bytes));
    if (cudaMallocFromPoolAsync(p, bytes, b->ctx->pool, b->st) != cudaSuccess) {
        cudaGetLastError();
        ctx_release(b->ctx, bytes);
        return fail(b->ctx, SOIL_ERR_OOM, "device allocation of %llu bytes failed",
                    (unsigned long long)bytes);
    }
    b->dev_bytes += bytes;
    return SOIL_OK;
}

void bfree(soil_batch* b, void* p, uint64_t bytes) {
    if (!p) return;
    cudaFreeAsync(p, b->st);  // after the batch's work already enqueued
    if (bytes == 0) bytes = 16;
    ctx_release(b->ctx, bytes);
    b->dev_bytes -= bytes;
}

enum { HT_INTEGRATE, HT_SORT, HT_BORDER_PLAN, HT_BORDERS, HT_NEIGHBOR, HT_LISTS, HT_WAIT };

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int wait(soil_batch* b) {
    b->waits += 1;
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t e = cudaStreamSynchronize(b->st);
    const double w = ms_since(t0);
    b->host_ms[HT_WAIT] += w;
    b->wait_pending_ms += w;
    BCK(e);
    return SOIL_OK;
}

// close a host planning section: its time since the last mark, waits excluded
void mark(soil_batch* b, int section) {
    const auto now = std::chrono::steady_clock::now();
    b->host_ms[section] += std::chrono::duration<double, std::milli>(now - b->hlast).count() -
                           b->wait_pending_ms;
    b->wait_pending_ms = 0.0;
    b->hlast = now;
}

// ---- stages -------------------------------------------------------------------
int stage_grow(soil_batch* b, Stage& g, size_t need) {
    if (need <= g.cap) return SOIL_OK;
    // every copy from the old buffer and every kernel reading the old device
    // region has to finish first
    TRY(wait(b));
    size_t ncap = std::max<size_t>(need + need / 2, 1u << 20);
    if (g.h) cudaFreeHost(g.h);
    if (g.d) bfree(b, g.d, g.cap);
    g.h = nullptr;
    g.d = nullptr;
    g.cap = 0;
    if (cudaMallocHost((void**)&g.h, ncap) != cudaSuccess) {
        cudaGetLastError();
        g.h = nullptr;
        return fail(b->ctx, SOIL_ERR_OOM, "pinned allocation of %zu bytes failed", ncap);
    }
    TRY(balloc(b, (void**)&g.d, ncap));
    g.cap = ncap;
    return SOIL_OK;
}

int stage_begin(soil_batch* b, Stage& g) {
    if (!g.ev) BCK(cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming));
    if (g.pending) BCK(cudaEventSynchronize(g.ev));
    g.pending = false;
    g.used = 0;
    g.nspans = 0;
    return SOIL_OK;
}

int stage_add(Stage& g) {
    if (g.nspans == g.spans.size()) g.spans.emplace_back();
    g.spans[g.nspans].clear();
    return (int)g.nspans++;
}

// Copy host bytes to a device address through the stage's pinned buffer.
int stage_put(soil_batch* b, Stage& g, void* dst, const void* src, size_t bytes) {
    if (!bytes) return SOIL_OK;
    const size_t off = (g.used + 15) & ~(size_t)15;
    if (off + bytes > g.cap) {
        TRY(stage_grow(b, g, off + bytes));
    }
    std::memcpy(g.h + off, src, bytes);
    BCK(cudaMemcpyAsync(dst, g.h + off, bytes, cudaMemcpyHostToDevice, b->st));
    g.used = off + bytes;
    g.pending = true;
    return SOIL_OK;
}

// Pack the stage's spans after its puts, upload them in one copy and fill
// g.out; records the stage event.
int stage_commit(soil_batch* b, Stage& g) {
    size_t off = (g.used + 15) & ~(size_t)15;
    const size_t first = off;
    std::vector<size_t> at(g.nspans);
    for (size_t k = 0; k < g.nspans; ++k) {
        const SpanBuild& s = g.spans[k];
        const size_t n = s.box.size();
        at[k] = off;
        off += (n + 1) * 8;
        off += ((n * 4) + 7) & ~(size_t)7;
        off += ((n * 4) + 7) & ~(size_t)7;
        off += (n + 7) & ~(size_t)7;
    }
    // puts already enqueued from this buffer finish inside stage_grow's wait;
    // their bytes were copied out by then, so a fresh buffer is safe
    if (off > g.cap) TRY(stage_grow(b, g, off));
    g.out.resize(g.nspans);
    for (size_t k = 0; k < g.nspans; ++k) {
        const SpanBuild& s = g.spans[k];
        const size_t n = s.box.size();
        size_t o = at[k];
        Span& sp = g.out[k];
        std::memcpy(g.h + o, s.start.data(), (n + 1) * 8);
        sp.start = (const uint64_t*)(g.d + o);
        o += (n + 1) * 8;
        std::memcpy(g.h + o, s.box.data(), n * 4);
        sp.box = (const uint32_t*)(g.d + o);
        o += ((n * 4) + 7) & ~(size_t)7;
        std::memcpy(g.h + o, s.base.data(), n * 4);
        sp.base = (const uint32_t*)(g.d + o);
        o += ((n * 4) + 7) & ~(size_t)7;
        std::memcpy(g.h + o, s.flag.data(), n);
        sp.flag = (const uint8_t*)(g.d + o);
        sp.nseg = (uint32_t)n;
        sp.total = s.start.back();
    }
    if (off > first)
        BCK(cudaMemcpyAsync(g.d + first, g.h + first, off - first, cudaMemcpyHostToDevice, b->st));
    g.used = off;
    BCK(cudaEventRecord(g.ev, b->st));
    g.pending = true;
    return SOIL_OK;
}

// ---- stage timers ---------------------------------------------------------------
enum { BT_INTEGRATE, BT_SORT, BT_BORDERS, BT_NEIGHBOR, BT_LISTS, BT_FORCE, BT_REVERSE, BT_STEP };

cudaEvent_t take_ev(soil_batch* b) {
    if (!b->ev_pool.empty()) {
        cudaEvent_t e = b->ev_pool.back();
        b->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

void tic(soil_batch* b) {
    if (!b->timing) return;
    b->open_a = take_ev(b);
    if (b->open_a) cudaEventRecord(b->open_a, b->st);
}

void toc(soil_batch* b, int stage) {
    if (!b->timing || !b->open_a) return;
    cudaEvent_t z = take_ev(b);
    if (!z) return;
    cudaEventRecord(z, b->st);
    b->timed.push_back({stage, b->open_a, z});
    b->open_a = nullptr;
}

void resolve_timers(soil_batch* b) {
    if (b->timed.empty()) return;
    cudaStreamSynchronize(b->st);
    for (auto& t : b->timed) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t.a, t.z) == cudaSuccess) {
            b->stage_ms[t.stage] += ms;
            b->stage_n[t.stage] += 1;
        } else {
            cudaGetLastError();
        }
        b->ev_pool.push_back(t.a);
        b->ev_pool.push_back(t.z);
    }
    b->timed.clear();
}

// ---- per-box tables -----------------------------------------------------------
int set_index(const BoxDev& d, const soil_sys* s) { return d.set[0].x == s->A.x ? 0 : 1; }

void fill_dev(soil_batch* b, uint32_t k) {
    const soil_sys* s = b->slot[k];
    const BoxDev& prev = b->h_dev[k];
    BoxDev d;
    std::memset(&d, 0, sizeof d);
    const bool swapped = prev.set[0].x != nullptr && prev.set[0].x == s->B.x &&
                         prev.set[1].x == s->A.x;
    std::memcpy(&d.set[0], swapped ? &s->B : &s->A, sizeof(AtomCols));
    std::memcpy(&d.set[1], swapped ? &s->A : &s->B, sizeof(AtomCols));
    d.set[0].pk = d.set[1].pk = nullptr;  // the batch's kernels read the columns
    d.radius_plane = s->cols[s->radius_col].plane0;
    d.shear_rate = s->shear_rate;
    d.yc = profile_center(s);
    d.lbx = s->lbx.p;
    d.lby = s->lby.p;
    d.lbz = s->lbz.p;
    d.sort_cell = s->sort_cell.p;
    d.sort_perm = s->sort_perm.p;
    d.sorted_local_cell = s->sorted_local_cell.p;
    d.cell_counts = s->cell_counts.p;
    d.cell_start = s->cell_start.p;
    d.cell_cursor = s->cell_cursor.p;
    d.atom_cell = s->atom_cell.p;
    d.sorted_atoms = s->sorted_atoms.p;
    d.asi = s->asi.p;
    d.rowcount = s->rowcount.p;
    d.row_slots = s->row_slots.p;
    d.offsets = s->offsets.p;
    d.indices = s->indices.p;
    d.sp = s->sp.p;
    d.spf = s->spf.p;
    d.in_count = s->in_count.p;
    d.in_start = s->in_start.p;
    d.in_cursor = s->in_cursor.p;
    d.in_list = s->in_list.p;
    d.ghost_root = s->ghost_root.p;
    d.ghost_chain = s->ghost_chain.p;
    for (int q = 0; q < kNumSwaps; ++q) d.send[q] = s->send[q].p;
    d.face_flags = s->face_flags.p;
    d.bcount = s->bcount.p;
    d.boff = s->boff.p;
    d.fold_start = s->fold_start.p;
    d.fold_list = s->fold_list.p;
    d.seq_cnt = s->seq_cnt.p;
    d.grp_cnt = s->grp_cnt.p;
    d.grp_start = s->grp_start.p;
    d.seq = s->seq.p;
    d.seq_owner = s->seq_owner.p;
    d.cap = s->acap;
    zero_planes_of(s, SOIL_COL_FORWARD, d.fwd.idx, &d.fwd.n);
    zero_planes_of(s, SOIL_COL_REVERSE, d.rev.idx, &d.rev.n);
    zero_planes_of(s, SOIL_COL_ZERO, d.zero.idx, &d.zero.n);
    if (std::memcmp(&d, &prev, sizeof d) != 0) {
        b->h_dev[k] = d;
        b->dev_dirty[k] = 1;
    }
}

// Per-step values of box k from its host state.  post_flip: the spatial sort
// of this step moves the columns to the other set.  bds: this step's border
// dims (NULL keeps the previous thresholds and takes the swap shifts of the
// last borders).
int fill_step(soil_batch* b, uint32_t k, bool post_flip, const BorderDim* bds) {
    const soil_sys* s = b->slot[k];
    BoxStep& t = b->h_step[k];
    const std::vector<int32_t>& sten = s->newton ? s->stencil_fwd : s->stencil;
    const std::vector<int32_t> runs = stencil_runs(sten, s->newton);
    if (runs.size() > (size_t)kMaxStencil)
        return fail(s->ctx, SOIL_ERR_INVALID,
                    "bin stencil of %zu cell runs exceeds the batched limit %d", runs.size() / 2,
                    kMaxStencil / 2);
    t.nlocal = s->nlocal;
    t.nghost = s->nghost;
    t.cur = set_index(b->h_dev[k], s);
    t.post = post_flip ? 1 - t.cur : t.cur;
    t.dt = s->dt;
    t.geom = geom_of(s);
    for (int d = 0; d < 3; ++d) t.bvel[d] = s->bvel[d];
    t.grid = grid_of(s);
    t.ncells = (uint32_t)s->total_cells;
    t.nstencil = (int32_t)(runs.size() / 2);
    t.pre_ranges = pairs_pre_ranges();
    std::memset(t.stencil, 0, sizeof t.stencil);
    if (!runs.empty()) std::memcpy(t.stencil, runs.data(), runs.size() * 4);
    t.has_self = s->stencil_self ? 1 : 0;
    t.newton = s->newton ? 1 : 0;
    t.uniform = s->has_uniform ? 1 : 0;
    t.filter = s->filter == SOIL_FILTER_FP32_RECHECK ? 1 : 0;
    t.cut_sq = s->uniform_cut_sq;
    t.sf_sq = s->skin_fraction * s->skin_fraction;
    t.sf = s->skin_fraction;
    t.eps32 = pair_eps(s);
    t.thr_sq = displacement_threshold_sq(s);
    for (int d = 0; d < 3; ++d) {
        t.box[d] = s->pbc_box[d];
        t.ibox[d] = 1.0 / s->pbc_box[d];  // ibx = 1.0 / bx (neighbor.rs:716-718)
    }
    if (bds) {
        for (int d = 0; d < 3; ++d) {
            t.thresh_lo[d] = bds[d].thresh_lo;
            t.thresh_hi[d] = bds[d].thresh_hi;
            for (int sw = 0; sw < 2; ++sw)
                for (int q = 0; q < 3; ++q) {
                    t.sc.off[2 * d + sw][q] = bds[d].shift[sw][q];
                    t.sc.voff[2 * d + sw][q] = bds[d].vshift[sw][q];
                }
        }
    } else {
        t.sc = swap_const(s);
    }
    t.K = s->harmonic_k;
    t.max_tiles = 0;
    t.segs_ok = pair_segments(sten, s->stencil_self, s->newton, &t.segs) ? 1 : 0;
    b->step_dirty[k] = 1;
    return SOIL_OK;
}

// Upload the changed rows of both tables, one copy per run of changed slots.
template <class T>
int put_dirty(soil_batch* b, Stage& g, std::vector<uint8_t>& dirty, const std::vector<T>& host,
              T* dev) {
    const uint32_t n = b->cap;
    uint32_t k = 0;
    while (k < n) {
        if (!dirty[k]) {
            ++k;
            continue;
        }
        uint32_t e = k + 1;
        // merge runs separated by short gaps
        while (e < n) {
            if (dirty[e]) {
                ++e;
                continue;
            }
            uint32_t f = e;
            while (f < n && !dirty[f] && f - e < 8) ++f;
            if (f < n && dirty[f]) e = f;
            else break;
        }
        TRY(stage_put(b, g, dev + k, host.data() + k, (size_t)(e - k) * sizeof(T)));
        for (uint32_t q = k; q < e; ++q) dirty[q] = 0;
        k = e;
    }
    return SOIL_OK;
}

int put_tables(soil_batch* b, Stage& g) {
    TRY(put_dirty(b, g, b->dev_dirty, b->h_dev, b->d_dev));
    TRY(put_dirty(b, g, b->step_dirty, b->h_step, b->d_step));
    return SOIL_OK;
}

BatchArgs args_of(const soil_batch* b) {
    BatchArgs a;
    a.dev = b->d_dev;
    a.step = b->d_step;
    a.flags = b->d_flags;
    a.bstate = b->d_bstate;
    a.totals = b->d_totals;
    return a;
}

int check_kernels(soil_batch* b) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(b->ctx, SOIL_ERR_CUDA, "batched kernel launch: %s", cudaGetErrorString(e));
    return SOIL_OK;
}

// ---- slot capacity --------------------------------------------------------------
int grow_slots(soil_batch* b, uint32_t need) {
    if (need <= b->cap) return SOIL_OK;
    TRY(wait(b));
    const uint32_t ncap = std::max<uint32_t>(need, std::max<uint32_t>(64u, b->cap * 2));
    BoxDev* nd = nullptr;
    BoxStep* ns = nullptr;
    DevFlags* nf = nullptr;
    uint32_t *nb = nullptr, *nt = nullptr;
    TRY(balloc(b, (void**)&nd, (uint64_t)ncap * sizeof(BoxDev)));
    TRY(balloc(b, (void**)&ns, (uint64_t)ncap * sizeof(BoxStep)));
    TRY(balloc(b, (void**)&nf, (uint64_t)ncap * sizeof(DevFlags)));
    TRY(balloc(b, (void**)&nb, (uint64_t)ncap * kBorderStateWords * 4));
    TRY(balloc(b, (void**)&nt, (uint64_t)ncap * 4));
    DevFlags* hf = nullptr;
    uint32_t *hb = nullptr, *ht = nullptr;
    if (cudaMallocHost((void**)&hf, (size_t)ncap * sizeof(DevFlags)) != cudaSuccess ||
        cudaMallocHost((void**)&hb, (size_t)ncap * kBorderStateWords * 4) != cudaSuccess ||
        cudaMallocHost((void**)&ht, (size_t)ncap * 4) != cudaSuccess) {
        cudaGetLastError();
        if (hf) cudaFreeHost(hf);
        if (hb) cudaFreeHost(hb);
        if (ht) cudaFreeHost(ht);
        return fail(b->ctx, SOIL_ERR_OOM, "pinned allocation failed");
    }
    bfree(b, b->d_dev, (uint64_t)b->cap * sizeof(BoxDev));
    bfree(b, b->d_step, (uint64_t)b->cap * sizeof(BoxStep));
    bfree(b, b->d_flags, (uint64_t)b->cap * sizeof(DevFlags));
    bfree(b, b->d_bstate, (uint64_t)b->cap * kBorderStateWords * 4);
    bfree(b, b->d_totals, (uint64_t)b->cap * 4);
    if (b->h_flags) cudaFreeHost(b->h_flags);
    if (b->h_bread) cudaFreeHost(b->h_bread);
    if (b->h_totals) cudaFreeHost(b->h_totals);
    b->d_dev = nd;
    b->d_step = ns;
    b->d_flags = nf;
    b->d_bstate = nb;
    b->d_totals = nt;
    b->h_flags = hf;
    b->h_bread = hb;
    b->h_totals = ht;
    b->slot.resize(ncap, nullptr);
    b->saved.resize(ncap, nullptr);
    BoxDev zd;
    std::memset(&zd, 0, sizeof zd);
    BoxStep zs;
    std::memset(&zs, 0, sizeof zs);
    b->h_dev.resize(ncap, zd);
    b->h_step.resize(ncap, zs);
    b->bds.resize(ncap);
    b->dev_dirty.assign(ncap, 0);
    b->step_dirty.assign(ncap, 0);
    for (uint32_t k = 0; k < b->cap; ++k)
        if (b->slot[k]) b->dev_dirty[k] = b->step_dirty[k] = 1;
    b->binit.assign((size_t)ncap * kBorderStateWords, 0u);
    for (auto* v : {&b->check, &b->full_at_pbc, &b->run, &b->periodic, &b->apply, &b->rebuild,
                    &b->planned})
        v->assign(ncap, 0);
    b->hot.resize(ncap);
    b->cap = ncap;
    return SOIL_OK;
}

// The staged pair count serves the batch when SOIL_PAIRS_STAGED=1.
bool pairs_staged_on() {
    const char* env = std::getenv("SOIL_PAIRS_STAGED");
    return env && std::atoi(env) != 0;  // measured slower: off unless asked
}

// ---- one step -------------------------------------------------------------------
int launch_borders(soil_batch* b, const std::vector<uint32_t>& R, Stage& g, bool retry) {
    TRY(stage_begin(b, g));
    TRY(put_tables(b, g));
    if (retry) std::memcpy(b->binit.data(), b->h_bread, (size_t)b->cap * kBorderStateWords * 4);
    // border state rows of the boxes in R start at zero
    uint32_t lo = b->cap, hi = 0;
    for (uint32_t k : R) {
        std::memset(b->binit.data() + (size_t)k * kBorderStateWords, 0, kBorderStateWords * 4);
        lo = std::min(lo, k);
        hi = std::max(hi, k + 1);
    }
    if (lo < hi)
        TRY(stage_put(b, g, b->d_bstate + (size_t)lo * kBorderStateWords,
                      b->binit.data() + (size_t)lo * kBorderStateWords,
                      (size_t)(hi - lo) * kBorderStateWords * 4));
    const int wt = stage_add(g);
    for (uint32_t k : R) g.spans[wt].add(k, (b->hot[k].nlocal + 31) / 32, 0);
    TRY(stage_commit(b, g));
    const BatchArgs a = args_of(b);
    tic(b);
    b_border_faces(b->st, g.out[wt], a);
    b_border_cat_scan(b->st, g.out[wt], a);
    b_border_images(b->st, g.out[wt], a);
    toc(b, BT_BORDERS);
    TRY(check_kernels(b));
    BCK(cudaMemcpyAsync(b->h_bread, b->d_bstate, (size_t)b->cap * kBorderStateWords * 4,
                        cudaMemcpyDeviceToHost, b->st));
    return wait(b);
}

// Host threads plan boxes in parallel; CUDA calls they make (allocations
// when a box grows) need the context's device current on that thread.
void bind_device(const soil_batch* b) {
    thread_local int bound = -1;
    if (bound != b->ctx->device) {
        cudaSetDevice(b->ctx->device);
        bound = b->ctx->device;
    }
}

// fn(k) for every slot k of `ks` on the host pool; first failure wins.
template <class F>
int for_boxes(soil_batch* b, const std::vector<uint32_t>& ks, F fn) {
    return b->pool->run(
        ks.size(),
        [&](size_t q) -> int {
            bind_device(b);
            return fn(ks[q]);
        },
        b->min_parallel);
}

int batch_step(soil_batch* b, bool last) {
    const std::vector<uint32_t>& M = b->members;
    const BatchArgs a = args_of(b);
    cudaStream_t st = b->st;

    // ---- deform, integrate (previous final fused in), displacement check ----
    b->hlast = std::chrono::steady_clock::now();
    b->wait_pending_ms = 0.0;
    Stage& g1 = b->stage[G_INTEGRATE];
    TRY(stage_begin(b, g1));
    TRY(put_tables(b, g1));
    const int sp_final = stage_add(g1), sp_prof = stage_add(g1), sp_init = stage_add(g1);
    bool any_check = false;
    for (uint32_t k : M) {
        soil_sys* s = b->slot[k];
        const bool profile_now = s->deform_initialized && s->shear && !s->shear_initialized;
        uint8_t fuse = s->pending_final ? 2 : 0;
        if (profile_now && s->pending_final) {
            g1.spans[sp_final].add_nz(k, s->nlocal, 0);
            fuse = 0;
        }
        if (deform_host(s)) g1.spans[sp_prof].add_nz(k, s->nlocal, 0);
        const bool check = s->state == COMMUNICATE_ONLY && displacement_needed(s);
        b->check[k] = check;
        any_check |= check;
        g1.spans[sp_init].add_nz(k, s->nlocal, 0, (uint8_t)((check ? 1 : 0) | fuse));
        s->pending_final = false;
    }
    TRY(stage_commit(b, g1));
    if (b->timing) {
        b->step_a = take_ev(b);
        if (b->step_a) cudaEventRecord(b->step_a, st);
    }
    tic(b);
    b_final(st, g1.out[sp_final], a);
    b_profile(st, g1.out[sp_prof], a);
    BCK(cudaMemsetAsync(b->d_flags, 0, (size_t)b->cap * sizeof(DevFlags), st));
    b_initial(st, g1.out[sp_init], a);
    toc(b, BT_INTEGRATE);
    TRY(check_kernels(b));
    if (any_check) {
        BCK(cudaMemcpyAsync(b->h_flags, b->d_flags, (size_t)b->cap * sizeof(DevFlags),
                            cudaMemcpyDeviceToHost, st));
        TRY(wait(b));
    }
    mark(b, HT_INTEGRATE);

    // ---- decide_rebuild, remove_ghosts, pbc, spatial sort ----
    TRY(for_boxes(b, M, [&](uint32_t k) -> int {
        soil_sys* s = b->slot[k];
        if (s->state == COMMUNICATE_ONLY) {
            const bool disp = b->check[k] && b->h_flags[k].rebuild != 0;
            if (needs_rebuild_with(s, disp)) s->state = FULL_REBUILD;
            else s->steps_since_build += 1;
        }
        b->full_at_pbc[k] = s->state == FULL_REBUILD;
        if (b->full_at_pbc[k]) s->nghost = 0;  // remove_ghost_atoms
        bool run, periodic;
        TRY(sort_plan(s, &run, &periodic));
        b->run[k] = run;
        b->periodic[k] = periodic;
        b->apply[k] = run && !periodic;
        // a box that rebuilds gets its border dims and neighbor parameters now,
        // so its step row is written once
        b->planned[k] = s->state == FULL_REBUILD;
        if (b->planned[k]) {
            border_setup(s, b->bds[k].data());
            neighbor_params(s);
        }
        if (run) fill_dev(b, k);
        if (run || b->planned[k])
            TRY(fill_step(b, k, b->apply[k] != 0, b->planned[k] ? b->bds[k].data() : nullptr));
        // host bookkeeping of a sort that always applies; the tables above
        // already describe the columns the kernels read and write
        if (run && !periodic) sort_done(s, true, false);
        auto& h = b->hot[k];
        h.cells = s->total_cells;
        if (b->full_at_pbc[k]) h.nghost = 0;
        b->rebuild[k] = s->state == FULL_REBUILD;
        return SOIL_OK;
    }));
    std::vector<uint32_t> S, I;
    bool any_pbc = false;
    for (uint32_t k : M) {
        any_pbc |= b->full_at_pbc[k] != 0;
        if (!b->run[k]) continue;
        S.push_back(k);
        if (b->periodic[k]) I.push_back(k);
    }
    if (any_pbc || !S.empty()) {
        Stage& g2 = b->stage[G_SORT];
        TRY(stage_begin(b, g2));
        TRY(put_tables(b, g2));
        const int s_pbc = stage_add(g2), s_cells = stage_add(g2), s_loc = stage_add(g2),
                  s_id = stage_add(g2), s_gather = stage_add(g2);
        for (uint32_t k : M)
            if (b->full_at_pbc[k]) g2.spans[s_pbc].add_nz(k, b->hot[k].nlocal, 0);
        for (uint32_t k : S) {
            const auto& h = b->hot[k];
            g2.spans[s_cells].add(k, h.cells, 0);
            g2.spans[s_loc].add_nz(k, h.nlocal, 0);
            if (b->periodic[k]) g2.spans[s_id].add_nz(k, h.nlocal, 0);
            if (b->apply[k]) g2.spans[s_gather].add_nz(k, h.nlocal, 0);
        }
        TRY(stage_commit(b, g2));
        tic(b);
        b_pbc(st, g2.out[s_pbc], a);
        b_zero_counts(st, g2.out[s_cells], a, BA_CELLS);
        b_cells(st, g2.out[s_loc], a, false);
        b_scan(st, g2.out[s_cells], a, BA_CELLS);
        b_scatter(st, g2.out[s_loc], a, false);
        b_segsort(st, g2.out[s_cells], a, BA_CELLS);
        b_permute_cells(st, g2.out[s_loc], a);
        b_identity(st, g2.out[s_id], a);
        b_perm_gather(st, g2.out[s_gather], a);
        toc(b, BT_SORT);
        TRY(check_kernels(b));
    }
    if (!I.empty()) {
        // periodic sorts apply only a permutation that is not the identity
        BCK(cudaMemcpyAsync(b->h_flags, b->d_flags, (size_t)b->cap * sizeof(DevFlags),
                            cudaMemcpyDeviceToHost, st));
        TRY(wait(b));
        Stage& g2b = b->stage[G_SORT_APPLY];
        TRY(stage_begin(b, g2b));
        const int s_gather = stage_add(g2b);
        for (uint32_t k : I) {
            b->apply[k] = b->h_flags[k].not_identity != 0;
            if (b->apply[k]) {
                TRY(fill_step(b, k, true, b->planned[k] ? b->bds[k].data() : nullptr));
                g2b.spans[s_gather].add_nz(k, b->hot[k].nlocal, 0);
            }
        }
        TRY(put_tables(b, g2b));
        TRY(stage_commit(b, g2b));
        b_perm_gather(st, g2b.out[s_gather], a);
        TRY(check_kernels(b));
    }
    for (uint32_t k : I) {  // periodic sorts: applied only when not the identity
        sort_done(b->slot[k], b->apply[k] != 0, true);
        b->rebuild[k] = b->slot[k]->state == FULL_REBUILD;
    }
    mark(b, HT_SORT);

    // ---- borders ----
    std::vector<uint32_t> R;
    for (uint32_t k : M)
        if (b->rebuild[k]) R.push_back(k);
    TRY(for_boxes(b, R, [&](uint32_t k) -> int {
        soil_sys* s = b->slot[k];
        s->nghost = 0;
        if (!b->planned[k]) {  // became a rebuild through its periodic sort
            border_setup(s, b->bds[k].data());
            neighbor_params(s);
        }
        TRY(borders_reserve(s));
        fill_dev(b, k);
        // the row needs rewriting when the columns moved (set order changed)
        if (!b->planned[k] || b->dev_dirty[k]) TRY(fill_step(b, k, false, b->bds[k].data()));
        return SOIL_OK;
    }));
    mark(b, HT_BORDER_PLAN);
    if (!R.empty()) {
        std::vector<uint32_t> todo = R;
        for (int attempt = 0;; ++attempt) {
            TRY(launch_borders(b, todo, b->stage[G_BORDERS], attempt > 0));
            std::vector<uint32_t> over;
            for (uint32_t k : todo)
                if (b->h_bread[(size_t)k * kBorderStateWords + 10]) over.push_back(k);
            if (over.empty()) break;
            if (attempt == 3) return fail(b->ctx, SOIL_ERR_CAPACITY, "ghost capacity did not converge");
            b->border_retries += over.size();
            TRY(for_boxes(b, over, [&](uint32_t k) -> int {
                soil_sys* s = b->slot[k];
                const uint32_t* hb = b->h_bread + (size_t)k * kBorderStateWords;
                TRY(grow_atoms(s, (uint64_t)hb[3] + 1024, s->nlocal));
                TRY(borders_arrays(s));
                fill_dev(b, k);
                return fill_step(b, k, false, b->bds[k].data());
            }));
            todo.swap(over);
        }
        mark(b, HT_BORDERS);
        TRY(for_boxes(b, R, [&](uint32_t k) -> int {
            soil_sys* s = b->slot[k];
            TRY(borders_done(s, b->h_bread + (size_t)k * kBorderStateWords, b->bds[k].data()));
            TRY(neighbor_plan(s));
            fill_dev(b, k);
            auto& h = b->hot[k];
            h.nghost = s->nghost;
            h.cells = s->total_cells;
            // local bins of this step's sort are reused once, by this build
            h.cells_valid = s->local_cells_valid ? 1 : 0;
            s->local_cells_valid = false;
            return SOIL_OK;
        }));
    }

    // ---- fold program, forward comm, neighbor build (pair count pass) ----
    Stage& g4 = b->stage[G_NEIGHBOR];
    TRY(stage_begin(b, g4));
    TRY(put_tables(b, g4));
    const int f_loc = stage_add(g4), s_fwd = stage_add(g4), n_cells = stage_add(g4),
              n_copy = stage_add(g4), n_bin = stage_add(g4), n_all = stage_add(g4),
              n_rows = stage_add(g4), n_tiles = stage_add(g4);
    for (uint32_t k : M) {
        const auto& h = b->hot[k];
        if (!b->rebuild[k]) {
            g4.spans[s_fwd].add_nz(k, h.nghost, 0);
            continue;
        }
        const uint64_t nl = h.nlocal, ng = h.nghost;
        g4.spans[f_loc].add_nz(k, nl, 0);
        g4.spans[n_cells].add(k, h.cells, 0);
        if (h.cells_valid) {
            g4.spans[n_copy].add_nz(k, nl, 0);
            g4.spans[n_bin].add_nz(k, ng, nl);
        } else {
            g4.spans[n_bin].add_nz(k, nl + ng, 0);
        }
        g4.spans[n_all].add_nz(k, nl + ng, 0);
        g4.spans[n_rows].add(k, nl, 0);
        g4.spans[n_tiles].add_nz(k, (nl + 31) / 32, 0);
    }
    TRY(stage_commit(b, g4));
    tic(b);
    b_forward(st, g4.out[s_fwd], a);
    if (!R.empty()) {
        b_save_positions(st, g4.out[f_loc], a);
        b_zero_counts(st, g4.out[n_cells], a, BA_NEIGH_CELLS);
        b_copy_count_local_cells(st, g4.out[n_copy], a);
        b_cells(st, g4.out[n_bin], a, true);
        b_scan(st, g4.out[n_cells], a, BA_NEIGH_CELLS);
        b_scatter(st, g4.out[n_all], a, true);
        b_segsort(st, g4.out[n_cells], a, BA_NEIGH_CELLS);
        b_sorted_views(st, g4.out[n_all], a);
        if (pairs_staged_on()) b_pairs_staged(st, g4.out[n_tiles], a);
        else b_pairs_rows(st, g4.out[f_loc], a);
        b_scan(st, g4.out[n_rows], a, BA_ROWS);
        toc(b, BT_NEIGHBOR);
        TRY(check_kernels(b));
        BCK(cudaMemcpyAsync(b->h_totals, b->d_totals, (size_t)b->cap * 4, cudaMemcpyDeviceToHost, st));
        BCK(cudaMemcpyAsync(b->h_flags, b->d_flags, (size_t)b->cap * sizeof(DevFlags),
                            cudaMemcpyDeviceToHost, st));
        TRY(wait(b));
        mark(b, HT_NEIGHBOR);
        TRY(for_boxes(b, R, [&](uint32_t k) -> int {
            soil_sys* s = b->slot[k];
            if (b->h_flags[k].error)
                return fail(b->ctx, SOIL_ERR_INVALID,
                            "neighbor stencil left the bin grid (atom outside the ghost layers)");
            const uint64_t np = b->h_totals[k], total = s->nlocal + s->nghost;
            TRY(ensure(s, s->indices, np + 1, 0, pair_room(np)));
            TRY(ensure(s, s->in_count, total + 1, 0, s->acap + 1));
            s->in_zero = 0;  // the batch's count pass leaves the counts behind
            TRY(ensure(s, s->in_start, total + 2, 0, s->acap + 2));
            TRY(ensure(s, s->in_cursor, total + 1, 0, s->acap + 1));
            TRY(ensure(s, s->in_list, np + 1, 0, pair_room(np)));
            const int fv = force_variant();
            if (s->few_images && fv != SOIL_FORCE_GATHER && fv != SOIL_FORCE_CSR) {
                // the grouped consumer's sequences, built this step
                TRY(ensure(s, s->seq_cnt, total + 1, 0, s->acap + 1));
                TRY(ensure(s, s->grp_cnt, s->nlocal + 1, 0, s->acap + 1));
                TRY(ensure(s, s->grp_start, s->nlocal + 2, 0, s->acap + 2));
                TRY(ensure(s, s->seq, 2 * np + 1, 0, 2 * pair_room(np)));
                TRY(ensure(s, s->seq_owner, 2 * np + 1, 0, 2 * pair_room(np)));
            }
            s->npairs = np;
            s->rebuilds += 1;
            s->in_lists_valid = true;
            s->seq_valid = false;  // set once this step's sequences are enqueued
            s->order_valid = false;
            s->split_valid = false;
            s->hflags->candidates = b->h_flags[k].candidates;
            s->hflags->rechecked = b->h_flags[k].rechecked;
            fill_dev(b, k);
            return SOIL_OK;
        }));
    }

    // ---- CSR fill, incoming lists, force, reverse comm, final ----
    Stage& g5 = b->stage[G_FORCE];
    std::vector<uint32_t> grouped_now;  // rebuilding boxes that build grouped sequences
    TRY(stage_begin(b, g5));
    TRY(put_tables(b, g5));
    const int r_loc = stage_add(g5), r_all = stage_add(g5), r_scan = stage_add(g5),
              h_all = stage_add(g5), v_loc = stage_add(g5), l_loc = stage_add(g5),
              q_all = stage_add(g5), q_grp = stage_add(g5), q_loc = stage_add(g5),
              t_tiles = stage_add(g5), t_walk = stage_add(g5);
    // Boxes whose locals have at most 7 images take the grouped consumer (its
    // sequences built at each rebuild, reverse comm folded in); the others the
    // per-atom gather and a reverse pass.
    grouped_now.clear();
    // The batch's consumer: the grouped kernels when SOIL_FORCE names one, else
    // the per-atom gather with a reverse pass (measured fastest on the
    // batched boxes, whose frequent rebuilds favour kernels without per-build
    // preparation).
    int variant = force_variant();
    if (variant == SOIL_FORCE_CSR) variant = SOIL_FORCE_GATHER;
    for (uint32_t k : M) {
        const auto& h = b->hot[k];
        const soil_sys* s = b->slot[k];
        const uint64_t nl = h.nlocal, total = nl + h.nghost;
        const bool grouped = variant != SOIL_FORCE_GATHER && s->few_images &&
                             (b->rebuild[k] || s->seq_valid);
        if (b->rebuild[k]) {
            g5.spans[r_loc].add_nz(k, nl, 0);
            g5.spans[r_all].add_nz(k, total, 0);
            g5.spans[r_scan].add(k, total, 0);
            if (grouped) {
                g5.spans[q_all].add_nz(k, total, 0);
                g5.spans[q_grp].add(k, nl, 0);
                g5.spans[q_loc].add_nz(k, nl, 0);
                grouped_now.push_back(k);
            }
        }
        if (grouped) {
            if (variant == SOIL_FORCE_WALK) g5.spans[t_walk].add_nz(k, nl, 0);
            else g5.spans[t_tiles].add_nz(k, (nl + 31) / 32, 0);
        } else {
            g5.spans[h_all].add_nz(k, total, 0);
            if (h.newton && h.nghost) g5.spans[v_loc].add_nz(k, nl, 0);
        }
        g5.spans[l_loc].add_nz(k, nl, 0);
    }
    toc(b, BT_NEIGHBOR);  // no-op when the rebuild path closed it
    TRY(stage_commit(b, g5));
    tic(b);
    if (!R.empty()) {
        b_pairs_fill(st, g5.out[r_loc], a);
        b_zero_counts(st, g5.out[r_scan], a, BA_IN);
        b_in_count(st, g5.out[r_loc], a);
        b_scan(st, g5.out[r_scan], a, BA_IN);
        b_in_scatter(st, g5.out[r_loc], a);
        b_segsort(st, g5.out[r_all], a, BA_IN);
        b_seq_count(st, g5.out[q_all], a);
        b_scan(st, g5.out[q_grp], a, BA_GRP);
        b_seq_fill(st, g5.out[q_loc], a);
        for (uint32_t k : grouped_now) b->slot[k]->seq_valid = true;
    }
    toc(b, BT_LISTS);
    tic(b);
    b_force_grouped(st, g5.out[t_tiles], a);
    b_force_walk(st, g5.out[t_walk], a);
    b_harmonic(st, g5.out[h_all], a);
    toc(b, BT_FORCE);
    tic(b);
    b_reverse(st, g5.out[v_loc], a);
    if (last) b_final(st, g5.out[l_loc], a);
    toc(b, BT_REVERSE);
    if (b->timing && b->step_a) {
        b->open_a = b->step_a;
        b->step_a = nullptr;
        toc(b, BT_STEP);
    }
    TRY(check_kernels(b));
    TRY(for_boxes(b, M, [&](uint32_t k) -> int {
        soil_sys* s = b->slot[k];
        s->pending_final = !last;
        s->steps_done += 1;
        return SOIL_OK;
    }));
    mark(b, HT_LISTS);
    b->steps += 1;
    return SOIL_OK;
}

// Occupied slots, largest box first: segment-per-CTA kernels then start the
// longest segments first.
void rebuild_members(soil_batch* b) {
    b->members.clear();
    for (uint32_t k = 0; k < b->cap; ++k)
        if (b->slot[k]) b->members.push_back(k);
    std::stable_sort(b->members.begin(), b->members.end(), [&](uint32_t x, uint32_t y) {
        return b->slot[x]->nlocal > b->slot[y]->nlocal;
    });
}

int detach(soil_batch* b, uint32_t k) {
    soil_sys* s = b->slot[k];
    s->counts_clean = 0;  // the batch's counting passes leave counts behind
    s->stencil_on_device.clear();
    s->pk_valid = false;  // the batch moved atoms without the packed records
    s->st = b->saved[k];
    // The batch leaves the last build's filter statistics in the host copy
    // only; on its own the system refreshes the host copy from the device one
    // (a displacement check's read-back), so that one gets them too.
    static_assert(offsetof(DevFlags, rechecked) == offsetof(DevFlags, candidates) + 8,
                  "DevFlags layout");
    if (cudaMemcpyAsync(&s->dflags->candidates, &s->hflags->candidates, 16,
                        cudaMemcpyHostToDevice, s->st) != cudaSuccess)
        cudaGetLastError();
    s->batch = nullptr;
    b->slot[k] = nullptr;
    b->saved[k] = nullptr;
    BoxDev zd;
    std::memset(&zd, 0, sizeof zd);
    b->h_dev[k] = zd;
    b->dev_dirty[k] = 0;
    b->step_dirty[k] = 0;
    return SOIL_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int soil_batch_create(soil_ctx* ctx, soil_batch** out) {
    if (!ctx || !out) return SOIL_ERR_INVALID;
    *out = nullptr;
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, SOIL_ERR_CUDA, "cudaSetDevice(%d) failed", ctx->device);
    }
    soil_batch* b = new (std::nothrow) soil_batch();
    if (!b) return SOIL_ERR_OOM;
    b->ctx = ctx;
    // planning threads: SOIL_HOST_THREADS, else up to 16 hardware threads
    int threads = (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (const char* e = std::getenv("SOIL_HOST_THREADS")) threads = std::max(1, std::atoi(e));
    if (const char* e = std::getenv("SOIL_HOST_MIN_PARALLEL"))
        b->min_parallel = (size_t)std::max(1, std::atoi(e));
    b->pool.reset(new HostPool(threads));
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return fail(ctx, SOIL_ERR_CUDA, "stream creation failed");
    }
    // every stage's staging buffers up front: a stage first used late (a
    // periodic sort that applies) then allocates nothing inside a run
    for (Stage& g : b->stage) {
        const int st = stage_grow(b, g, 1);
        if (st != SOIL_OK) {
            soil_batch_destroy(b);
            return st;
        }
    }
    *out = b;
    return SOIL_OK;
}

int soil_batch_destroy(soil_batch* b) {
    if (!b) return SOIL_OK;
    cudaStreamSynchronize(b->st);
    resolve_timers(b);
    for (cudaEvent_t e : b->ev_pool) cudaEventDestroy(e);
    if (b->open_a) cudaEventDestroy(b->open_a);
    if (b->step_a) cudaEventDestroy(b->step_a);
    for (uint32_t k = 0; k < b->cap; ++k)
        if (b->slot[k]) detach(b, k);
    for (Stage& g : b->stage) {
        if (g.h) cudaFreeHost(g.h);
        if (g.d) bfree(b, g.d, g.cap);
        if (g.ev) cudaEventDestroy(g.ev);
    }
    bfree(b, b->d_dev, (uint64_t)b->cap * sizeof(BoxDev));
    bfree(b, b->d_step, (uint64_t)b->cap * sizeof(BoxStep));
    bfree(b, b->d_flags, (uint64_t)b->cap * sizeof(DevFlags));
    bfree(b, b->d_bstate, (uint64_t)b->cap * kBorderStateWords * 4);
    bfree(b, b->d_totals, (uint64_t)b->cap * 4);
    if (b->h_flags) cudaFreeHost(b->h_flags);
    if (b->h_bread) cudaFreeHost(b->h_bread);
    if (b->h_totals) cudaFreeHost(b->h_totals);
    cudaStreamDestroy(b->st);
    delete b;
    return SOIL_OK;
}

int soil_batch_add(soil_batch* b, soil_sys* s) {
    if (!b || !s) return SOIL_ERR_INVALID;
    if (s->ctx != b->ctx) return fail(b->ctx, SOIL_ERR_INVALID, "system belongs to another context");
    if (s->batch) return fail(b->ctx, SOIL_ERR_STATE, "system is already batched");
    if (!s->setup_done) return fail(b->ctx, SOIL_ERR_STATE, "soil_sys_setup has not run");
    if (s->nlocal == 0) return fail(b->ctx, SOIL_ERR_INVALID, "a batched system needs atoms");
    if (!builtin_consumer(s))
        return fail(b->ctx, SOIL_ERR_INVALID,
                    "a batched system uses the built-in harmonic consumer and no force hook");
    if (s->slot_max) return fail(b->ctx, SOIL_ERR_INVALID, "a batched system has no neighbor slots");
    if (has_axis_deform(s))
        return fail(b->ctx, SOIL_ERR_INVALID, "a batched system has no orthogonal deform");
    if (pbc_mask(s) != 7) return fail(b->ctx, SOIL_ERR_INVALID, "a batched system is periodic");
    int zp[kMaxPlanes], nz;
    zero_planes_of(s, SOIL_COL_ZERO, zp, &nz);
    if (nz) return fail(b->ctx, SOIL_ERR_INVALID, "#[zero] columns are not supported in a batch");
    const std::vector<int32_t> runs =
        stencil_runs(s->newton ? s->stencil_fwd : s->stencil, s->newton);
    if (runs.size() > (size_t)kMaxStencil)
        return fail(b->ctx, SOIL_ERR_INVALID,
                    "bin stencil of %zu cell runs exceeds the batched limit %d", runs.size() / 2,
                    kMaxStencil / 2);
    BCK(cudaStreamSynchronize(s->st));
    TRY(wait(b));
    uint32_t k = 0;
    while (k < b->cap && b->slot[k]) ++k;
    if (k == b->cap) TRY(grow_slots(b, b->cap + 1));
    b->slot[k] = s;
    b->saved[k] = s->st;
    s->st = b->st;
    s->batch = b;
    std::memset(&b->h_dev[k], 0, sizeof(BoxDev));
    fill_dev(b, k);
    b->dev_dirty[k] = 1;
    b->hot[k].nlocal = s->nlocal;
    b->hot[k].nghost = s->nghost;
    b->hot[k].cells = s->total_cells;
    b->hot[k].newton = s->newton ? 1 : 0;
    b->hot[k].cells_valid = 0;
    TRY(fill_step(b, k, false, nullptr));
    rebuild_members(b);
    return SOIL_OK;
}

int soil_batch_remove(soil_batch* b, soil_sys* s) {
    if (!b || !s) return SOIL_ERR_INVALID;
    if (s->batch != b) return fail(b->ctx, SOIL_ERR_INVALID, "system is not in this batch");
    TRY(wait(b));
    for (uint32_t k = 0; k < b->cap; ++k)
        if (b->slot[k] == s) detach(b, k);
    rebuild_members(b);
    return SOIL_OK;
}

int soil_batch_size(soil_batch* b, uint32_t* n) {
    if (!b || !n) return SOIL_ERR_INVALID;
    *n = (uint32_t)b->members.size();
    return SOIL_OK;
}

int soil_batch_step(soil_batch* b, uint64_t nsteps) {
    if (!b) return SOIL_ERR_INVALID;
    if (b->members.empty()) return SOIL_OK;
    BCK(cudaSetDevice(b->ctx->device));
    for (uint64_t t = 0; t < nsteps; ++t) TRY(batch_step(b, t + 1 == nsteps));
    return SOIL_OK;
}

int soil_batch_sync(soil_batch* b) {
    if (!b) return SOIL_ERR_INVALID;
    return wait(b);
}

int soil_batch_stream(soil_batch* b, void** out) {
    if (!b || !out) return SOIL_ERR_INVALID;
    *out = (void*)b->st;
    return SOIL_OK;
}

int soil_batch_set_timing(soil_batch* b, int32_t on) {
    if (!b) return SOIL_ERR_INVALID;
    resolve_timers(b);
    b->timing = on != 0;
    for (int t = 0; t < SOIL_BATCH_NUM_TIMERS; ++t) {
        b->stage_ms[t] = 0.0;
        b->stage_n[t] = 0;
    }
    for (int t = 0; t < SOIL_BATCH_NUM_HOST_TIMERS; ++t) b->host_ms[t] = 0.0;
    return SOIL_OK;
}

int soil_batch_get_timing(soil_batch* b, double* ms, uint64_t* intervals) {
    if (!b) return SOIL_ERR_INVALID;
    resolve_timers(b);
    for (int t = 0; t < SOIL_BATCH_NUM_TIMERS; ++t) {
        if (ms) ms[t] = b->stage_ms[t];
        if (intervals) intervals[t] = b->stage_n[t];
    }
    return SOIL_OK;
}

int soil_batch_get_host_timing(soil_batch* b, double* ms) {
    if (!b || !ms) return SOIL_ERR_INVALID;
    for (int t = 0; t < SOIL_BATCH_NUM_HOST_TIMERS; ++t) ms[t] = b->host_ms[t];
    return SOIL_OK;
}

int soil_batch_stats(soil_batch* b, uint64_t* steps, uint64_t* host_waits, uint64_t* device_bytes,
                     uint64_t* border_retries) {
    if (!b) return SOIL_ERR_INVALID;
    if (steps) *steps = b->steps;
    if (host_waits) *host_waits = b->waits;
    if (device_bytes) *device_bytes = b->dev_bytes;
    if (border_retries) *border_retries = b->border_retries;
    return SOIL_OK;
}

}  // extern "C"
