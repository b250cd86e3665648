// sys_internal.cuh — host-side state of one system (the reference's Atom,
// Domain, Neighbor and CommTopology resources) and the helpers that the
// single-system entry points and the batch engine share.
#pragma once

#include <cfloat>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"

using namespace soil;

struct soil_ctx {
    int device = 0;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    std::string err;
    uint64_t allocs = 0, frees = 0;
    cudaMemPool_t pool = nullptr;  // stream-ordered device memory of every system and batch
    mutable std::mutex mu;  // guards in_use, the counters and err
};

namespace soil_host {

enum { FULL_REBUILD = SOIL_FULL_REBUILD, COMMUNICATE_ONLY = SOIL_COMMUNICATE_ONLY };

struct ColMeta {
    std::string name;
    int width;
    unsigned flags;
    int plane0;
};

template <class T>
struct DArr {
    T* p = nullptr;
    uint64_t cap = 0;  // elements
};

struct SwapHost {
    uint64_t recv_start = 0, recv_count = 0;
    uint64_t send_count = 0;  // recv_count, or the packed atoms of a swap with no neighbor
    double off[3] = {0, 0, 0};
    double voff[3] = {0, 0, 0};
};

}  // namespace soil_host

using soil_host::ColMeta;
using soil_host::DArr;
using soil_host::SwapHost;

struct soil_sys {
    soil_ctx* ctx = nullptr;
    cudaStream_t st = nullptr;
    double dt = 1.0;

    // ---- Domain (domain.rs:105-142), one rank ----
    double blo[3], bhi[3], size[3], sub_lo[3], sub_hi[3], sub_len[3];
    double sub_lam_lo[3] = {0, 0, 0}, sub_lam_hi[3] = {1, 1, 1};
    double tilt[3] = {0, 0, 0}, bvel[3] = {0, 0, 0};
    bool triclinic = false, bounds_changed = false;
    double domain_ghost_cutoff = 0.0;

    // ---- Neighbor scalars (neighbor.rs:87-174) ----
    double skin_fraction = 1.0, bin_min_size = 1.0, additive_skin = 0.0;
    uint64_t every = 0, sort_every = 1000;
    bool check = true, newton = true;
    int filter = SOIL_FILTER_FP64;
    double bin_size[3] = {1, 1, 1}, bin_origin[3] = {0, 0, 0};
    int32_t bin_count[3] = {1, 1, 1};
    uint64_t total_cells = 0;
    std::vector<int32_t> stencil, stencil_fwd;
    bool stencil_self = false;
    double pbc_box[3] = {0, 0, 0};
    double ghost_cutoff = 0.0, cached_min_skin = DBL_MAX, cached_max_cutoff = 0.0;
    bool has_uniform = false;
    double uniform_cut_sq = 0.0;
    uint64_t steps_since_build = 0, sort_counter = 0;
    bool local_cells_valid = false;
    uint64_t last_build_n = 0;  // last_build_pos.len()
    double cut_min_local = DBL_MAX, cut_max_local = -DBL_MAX;

    // ---- Atom counts / CommState ----
    uint64_t nlocal = 0, nghost = 0, npairs = 0;
    int state = soil_host::FULL_REBUILD;
    SwapHost swaps[kNumSwaps];
    int nswaps = 0;

    // ---- deform / consumer ----
    bool shear = false, shear_initialized = false, deform_initialized = false;
    // orthogonal deform per axis (style SOIL_DEFORM_*; lo0/hi0 set at setup)
    struct AxisDeform {
        int32_t style = 0;
        double a = 0.0, b = 0.0;
        uint64_t stage_steps = 0;
        double lo0 = 0.0, hi0 = 0.0;
    } axis[3];
    bool remap = true;
    // BoundaryType per axis (SOIL_BOUNDARY_*) and the shrink-wrap padding
    int32_t btype[3] = {SOIL_BOUNDARY_PERIODIC, SOIL_BOUNDARY_PERIODIC, SOIL_BOUNDARY_PERIODIC};
    double shrink_padding = 0.0;
    DArr<uint32_t> sel_flag, sel_pos, sel_out, sel_cnt;  // ordered selection scratch
    DArr<unsigned long long> ext;                        // shrink-wrap extent keys
    DArr<uint32_t> fold_roots, fold_nroots;  // locals with images (reverse comm), their count
    // border passes so far, the pass fold_roots belongs to, and the pass the
    // last reverse comm folded
    uint64_t border_gen = 0, fold_roots_gen = ~0ull, reverse_gen = ~0ull;
    double shear_rate = 0.0;
    uint64_t deform_step = 0;
    double harmonic_k = 0.0;
    int radius_col = -1;
    soil_force_fn hook = nullptr;
    void* hook_user = nullptr;
    bool in_lists_valid = false;

    // ---- columns ----
    std::vector<ColMeta> cols;
    int nplanes = 0;

    // ---- device memory ----
    uint64_t acap = 0;
    AtomCols A{}, B{};
    DArr<double> lbx, lby, lbz;
    DArr<uint32_t> sort_cell, sort_perm, sorted_local_cell;
    DArr<uint32_t> sort_start;  // the spatial sort's cell starts (its locals' bins)
    DArr<uint32_t> ghost_tmp;   // the neighbor build's unordered ghost slots
    DArr<uint32_t> cell_counts, cell_start, cell_cursor;
    // cell_counts[0, counts_clean) is known to be zero (the consuming scatters
    // leave it so); counts_at: the allocation that holds
    uint64_t counts_clean = 0;
    // in_count[0, in_zero) is known to be zero (pass 2 of the pair build
    // consumes the counts of pass 1); in_zero_at: the array it describes
    uint64_t in_zero = 0;
    const uint32_t* in_zero_at = nullptr;
    const uint32_t* counts_at = nullptr;
    std::vector<int32_t> stencil_on_device;  // the stencil last uploaded to d_stencil
    DArr<uint32_t> atom_cell, sorted_atoms, asi, rowcount, offsets, indices, row_slots;
    DArr<double4> sp;
    // persistent per-neighbor slots (slot_max == 0: disabled); buffer
    // slot_old holds the slots the last hook call wrote
    uint32_t slot_max = 0, slot_width = 0;
    DArr<uint32_t> slot_tag[2];
    DArr<double> slot_val[2];
    int slot_old = 0;
    DArr<float4> spf;
    DArr<uint32_t> in_count, in_start, in_cursor, in_list;
    DArr<uint32_t> in_split;  // per atom: transposed-list entries below it
    bool split_valid = false;
    // packed (x, y, z, r) records of the consumer kernels (AtomCols::pk);
    // pk_valid: they match the columns of every local and ghost
    DArr<double> pk;
    bool pk_valid = false;
    bool view_out = false;  // a device view was handed out since the last rebuild
    bool forces_dead = false;  // inside a step whose consumer overwrites every force
    // a border pass whose totals (hword + kBorderStateWords) are read back at
    // the following neighbor build's synchronisation, and its dims
    bool borders_pending = false;
    BorderDim pending_bds[3];
    // grouped partner sequences of the built-in consumer (rebuilt with the
    // lists): per-atom lengths, per-root group lengths and starts, entries
    DArr<uint32_t> seq_cnt, grp_cnt, grp_start, seq;
    DArr<uint8_t> seq_owner;
    bool seq_valid = false;
    bool few_images = false;  // no local has images on both sides of a dim (<= 7 images)
    DArr<uint32_t> rstate;    // resident steps: grid barrier words, step count, trip flag
    DArr<uint32_t> scan1p;    // single-pass scan: tile counter and descriptors (zeroed at growth)
    DArr<uint32_t> root_order;  // CSR-walk consumer: roots by work per block (rebuilt with the lists)
    bool order_valid = false;
    DArr<uint32_t> ghost_root, ghost_chain;
    DArr<uint32_t> fold_start, fold_list;  // reverse-comm fold program (written by borders)
    DArr<uint32_t> send[kNumSwaps];
    DArr<uint32_t> bstate;
    DArr<uint32_t> bcount, boff;  // per-warp chain-category counts / offsets of borders
    DArr<uint8_t> face_flags;
    uint64_t last_nghost = 0;
    DArr<uint32_t> scan_tmp;
    DArr<int32_t> d_stencil;
    DArr<double> stage;  // host-layout staging for uploads/downloads
    DArr<double*> d_colptrs;
    bool colptrs_dirty = true;  // d_colptrs no longer matches A (refreshed by make_view)
    DevFlags* dflags = nullptr;
    DevFlags* hflags = nullptr;  // pinned mirror
    uint32_t* hword = nullptr;   // pinned scratch words
    // the same two buffers as the device addresses them (mapped host memory):
    // kernels that end a phase write the host's words directly
    DevFlags* hflags_dev = nullptr;
    uint32_t* hword_dev = nullptr;

    // ---- phase timers ----
    struct TimedSpan {
        int timer;
        cudaEvent_t a, b;
        uint64_t launches;
    };
    uint32_t timing_mask = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<TimedSpan> spans;
    double timer_ms[SOIL_NUM_TIMERS] = {};
    uint64_t timer_launches[SOIL_NUM_TIMERS] = {};
    uint64_t timer_intervals[SOIL_NUM_TIMERS] = {};
    int open_timer = -1;
    cudaEvent_t open_ev = nullptr;
    cudaEvent_t ev_counts = nullptr;  // the pair build's counts are on the host
    uint64_t open_launches = 0;

    // ---- bookkeeping ----
    soil_batch* batch = nullptr;  // batch this system is stepped in (its stream is the batch's)
    bool setup_done = false, perm_valid = false, pending_final = false;
    uint64_t steps_done = 0, rebuilds = 0, sorts = 0;
};


namespace soil_host {

int fail(soil_ctx* ctx, int status, const char* fmt, ...);

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(s->ctx, SOIL_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                  \
    } while (0)

#define TRY(call)                        \
    do {                                 \
        int r_ = (call);                 \
        if (r_ != SOIL_OK) return r_;    \
    } while (0)

int ctx_reserve(soil_ctx* ctx, uint64_t bytes);
void ctx_release(soil_ctx* ctx, uint64_t bytes);
int dev_alloc(soil_sys* s, void** p, uint64_t bytes);
void dev_free(soil_sys* s, void* p, uint64_t bytes);

// Grow `a` to hold `need` elements; the first `keep` elements survive.  A
// new array gets room for `room` elements (at least need + 25%), so counts
// that drift between rebuilds (pairs, bins) can be given more headroom than
// the check itself.
template <class T>
int ensure(soil_sys* s, DArr<T>& a, uint64_t need, uint64_t keep = 0, uint64_t room = 0) {
    if (need <= a.cap && a.p) return SOIL_OK;
    uint64_t ncap = need + need / 4 + 64;
    if (room > ncap) ncap = room;
    void* np = nullptr;
    TRY(dev_alloc(s, &np, ncap * sizeof(T)));
    if (a.p && keep) CK(cudaMemcpyAsync(np, a.p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s->st));
    if (a.p) dev_free(s, a.p, a.cap * sizeof(T));  // stream-ordered, after the copy
    a.p = (T*)np;
    a.cap = ncap;
    return SOIL_OK;
}

int grow_atoms(soil_sys* s, uint64_t need, uint64_t keep);
int slots_grow(soil_sys* s, uint64_t cap, uint64_t keep);
// Room for arrays indexed by pair (CSR indices, incoming lists): pair counts
// drift between rebuilds, so a new array takes twice the current count.
inline uint64_t pair_room(uint64_t np) { return 2 * np + 1024; }
int update_colptrs(soil_sys* s);
bool deform_host(soil_sys* s);
int deform_step(soil_sys* s, bool* profile, RemapSpec* r);
bool has_axis_deform(const soil_sys* s);
int pbc_mask(const soil_sys* s);  // bit d: axis d periodic
double profile_center(const soil_sys* s);
int sort_plan(soil_sys* s, bool* run, bool* periodic);
void sort_done(soil_sys* s, bool apply, bool periodic);
void border_setup(const soil_sys* s, BorderDim bds[3]);
int borders_reserve(soil_sys* s);
int borders_arrays(soil_sys* s);
int borders_done(soil_sys* s, const uint32_t* hb, const BorderDim bds[3]);
void neighbor_params(soil_sys* s);
int neighbor_plan(soil_sys* s);
float pair_eps(const soil_sys* s);
bool pair_segments(const std::vector<int32_t>& sten, bool has_self, bool newton, PairSegs* sg);
int sync(soil_sys* s);
int check_launch(soil_sys* s);
// cell_counts[0, nc) zero before a counting pass
int counts_zero(soil_sys* s, uint64_t nc);
// The pair scan's stencil: offsets (ascending) merged into runs of consecutive
// cells, as (offset, cells) pairs; without newton the own cell (offset 0),
// which the scan takes first, is left out.
std::vector<int32_t> stencil_runs(const std::vector<int32_t>& sten, bool newton);
// Whether the pair scan preloads its ranges (SOIL_PAIRS_PRE=0: off; read at each call).
int pairs_pre_ranges();
// exclusive scan of in[0, n) into out[0, n] in one launch, errors into the
// system's device flags
int scan_1p(soil_sys* s, const uint32_t* in, uint32_t* out, uint64_t n);
Geom geom_of(const soil_sys* s);
Grid grid_of(const soil_sys* s);
void compute_bin_grid(soil_sys* s);
double displacement_threshold_sq(const soil_sys* s);
void zero_planes_of(const soil_sys* s, unsigned flag, int* out, int* n);
bool builtin_consumer(const soil_sys* s);
bool needs_rebuild_with(const soil_sys* s, bool disp);
bool displacement_needed(const soil_sys* s);
SwapConst swap_const(const soil_sys* s);
constexpr int kRowSlotsPerAtom = 16;
// Largest system that takes the device-resident light steps by default
// (SOIL_RESIDENT_STEPS=1 forces them on at any size, 0 off).
constexpr uint64_t kResidentAutoMaxAtoms = 1ull << 20;
// largest count the single-pass scan serves (scan_1p)
constexpr uint64_t kScan1pMaxCounts = 64ull * 2048ull;

}  // namespace soil_host
