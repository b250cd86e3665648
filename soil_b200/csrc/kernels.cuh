// kernels.cuh — launch wrappers of the soil_b200 CUDA kernels.
// Each wrapper enqueues on `st` and returns immediately.
#pragma once

#include <atomic>

#include "soil_internal.cuh"

namespace soil {

// Grid for a grid-stride kernel: per_sm CTAs on each of the 148 SMs, never
// more than the work needs.
unsigned grid_for(uint64_t n, int block = kBlock, int per_sm = 8);

// Grid of exactly one resident wave of kernel K (its CTAs per SM at kBlock
// threads and `smem` bytes of dynamic shared memory, queried once), never more
// than the work needs.  A grid-stride kernel launched with more CTAs than fit
// at once runs a partial second wave after the first (1,184 CTAs of a kernel
// that fits 6 per SM take two wave times for 1.33 waves of work).
template <auto K>
unsigned grid_wave(uint64_t n, size_t smem = 0) {
    static std::atomic<int> per_sm{0};
    int r = per_sm.load(std::memory_order_relaxed);
    if (r == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, K, kBlock, smem) != cudaSuccess ||
            r < 1) {
            cudaGetLastError();
            r = 8;
        }
        per_sm.store(r, std::memory_order_relaxed);
    }
    return grid_for(n, kBlock, r);
}

// Process-wide count of kernel launches issued by this library.
void note_launch();
uint64_t launches_so_far();

// ---- programmatic dependent launch ------------------------------------------
// The kernels of a step follow one another in one stream.  Every kernel
// launched with pdl_launch starts with pdl_wait(), before it touches global
// memory: the wait returns once the kernel before it in the stream has
// completed and its writes are visible (a no-op for a launch without the
// attribute).  Right after it, the kernel allows its own dependent to launch,
// so the dependent's launch and CTA set-up overlap this kernel's run and
// drain instead of following its completion; the dependent's CTAs take SM
// slots only as they free up and wait there.  A dependent can launch only
// once every CTA of this kernel has started, so this kernel's CTAs never wait
// for slots held by it (no deadlock, whatever the grid sizes).  SOIL_PDL=0
// launches plainly (read once).
__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
bool pdl_on();
template <class... E, class... A>
void pdl_launch(void (*k)(E...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_on() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(args)...);
}

// ---- integrate (k_integrate.cu) -------------------------------------------
// The displacement check fused into the integration pass (decide_rebuild's
// displacement_exceeded): last-build positions, threshold, periodic box.
struct CheckArgs {
    const double* lbx;
    const double* lby;
    const double* lbz;
    uint64_t n_check;
    double thr_sq;
    double box[3];
    double ibox[3];
    DevFlags* flags;
    int mask;  // periodic axes (7: fully periodic fast path)
};
CheckArgs make_check(const double* lbx, const double* lby, const double* lbz, uint64_t n_check,
                     double thr_sq, const double box[3], DevFlags* flags, int mask);
// forward_comm fused into the integration pass: every local writes its ghost
// images (fold program of the last border pass) from its new position and
// velocity, with the #[forward] planes; zero_ghost_force clears their forces.
struct FwdArgs {
    const uint32_t* fold_start;
    const uint32_t* fold_list;
    const uint32_t* chain;
    SwapConst sc;
    PlaneList fwd;
    int zero_ghost_force;
};
// initial_integration (+ optional fused force zeroing, displacement check
// and forward comm).  pbc_mask: bit d set for a periodic axis d (7: the
// fully periodic test).  fw NULL: no forward comm.
void launch_initial(cudaStream_t st, uint64_t n, const AtomCols& c, double dt, bool zero_force,
                    const double* lbx, const double* lby, const double* lbz, uint64_t n_check,
                    double thr_sq, const double box[3], DevFlags* flags, int pbc_mask = 7,
                    const FwdArgs* fw = nullptr);
// final_integration
void launch_final(cudaStream_t st, uint64_t n, const AtomCols& c, double dt);
// final_integration of step t fused with initial_integration of step t+1
void launch_final_initial(cudaStream_t st, uint64_t n, const AtomCols& c, double dt,
                          bool zero_force, const double* lbx, const double* lby,
                          const double* lbz, uint64_t n_check, double thr_sq,
                          const double box[3], DevFlags* flags, int pbc_mask = 7,
                          const FwdArgs* fw = nullptr);
// zero_all_forces over [0, n) + the #[zero] planes
void launch_zero_forces(cudaStream_t st, uint64_t n, const AtomCols& c, const int* zero_planes,
                        int nzero);
// pbc (orthogonal) / pbc_triclinic over locals
void launch_pbc(cudaStream_t st, uint64_t nlocal, const AtomCols& c, const Geom& g,
                const double bvel[3]);
// soil_deform first-step streaming profile vx += rate*(y - yc)
void launch_shear_profile(cudaStream_t st, uint64_t n, const AtomCols& c, double rate, double yc);

// Affine position remap of an orthogonal deform step: for each of the n
// listed dims, x_d = new_center + (x_d - old_center) * scale.
struct RemapSpec {
    int n = 0;
    int dim[3];
    double old_center[3], new_center[3], scale[3];
};
void launch_remap(cudaStream_t st, uint64_t n, const AtomCols& c, const RemapSpec& r);
// displacement_exceeded over [0, n) into flags->rebuild
void launch_disp_check(cudaStream_t st, uint64_t n, const AtomCols& c, const double* lbx,
                       const double* lby, const double* lbz, double thr_sq, const double box[3],
                       DevFlags* flags, int pbc_mask = 7);

// ---- non-periodic boundaries (k_bounds.cu) ---------------------------------
struct BoundsArgs {
    double lo[3], hi[3], size[3];
    int periodic;  // bit d: axis d is periodic
    Geom geom;     // triclinic boxes wrap and test in lamda space
    double bvel[3];
};
// pbc with fixed axes: wrap periodic axes, gone[i] = 1 for atoms to remove
void launch_pbc_bounded(cudaStream_t st, uint64_t n, const AtomCols& c, const BoundsArgs& b,
                        uint32_t* gone);
// flag[i] = v < thresh (side 0) or v >= thresh (side 1), i in [0, n), v the
// dim coordinate (lamda when triclinic)
void launch_face_flag(cudaStream_t st, uint64_t n, const AtomCols& c, const Geom& g, int dim,
                      double thresh, int side, uint32_t* flag);
// out[0..k) = the i with flag[i] != 0, ascending; pos[0..n] the exclusive
// scan of flag (pos[n] = k); temp holds scan_temp_words(n) u32
void launch_select(cudaStream_t st, uint64_t n, const uint32_t* flag, uint32_t* pos,
                   uint32_t* temp, uint32_t* out);
// ext[d] / ext[3 + d]: order keys of the min / max of x_d over [0, n), axes
// in mask (ext preset to all ones / zeros)
void launch_extent(cudaStream_t st, uint64_t n, const AtomCols& c, int mask,
                   unsigned long long* ext);
// inv[i] = 1.0 / m[i], i < n
void launch_inverse(cudaStream_t st, uint64_t n, const double* m, double* inv);
// pk[4 i .. 4 i + 3] = (x, y, z, rad) of atoms [0, n)
void launch_pack(cudaStream_t st, uint64_t n, const AtomCols& c, const double* rad, double* pk);
// host-layout conversions ([n][3] or [n][w] interleaved <-> SoA planes)
void launch_deinterleave3(cudaStream_t st, uint64_t n, const double* src, double* a, double* b,
                          double* c);
void launch_interleave3(cudaStream_t st, uint64_t n, double* dst, const double* a, const double* b,
                        const double* c);
void launch_interleave3i(cudaStream_t st, uint64_t n, int32_t* dst, const int32_t* a,
                         const int32_t* b, const int32_t* c);
void launch_deinterleave_w(cudaStream_t st, uint64_t n, int w, const double* src, double* dst0,
                           uint64_t cap);
void launch_interleave_w(cudaStream_t st, uint64_t n, int w, double* dst, const double* src0,
                         uint64_t cap);

// ---- scan (k_scan.cu) -----------------------------------------------------
// Exclusive scan: out[0..n] with out[n] = total.  `temp` holds
// scan_temp_words(n) u32.
uint64_t scan_temp_words(uint64_t n);
void exclusive_scan_u32(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n,
                        uint32_t* temp);
// Two independent scans in the same two launches (when each fits the
// two-launch form; else one after the other).  temp holds
// scan_temp_words(n0) + scan_temp_words(n1) u32.
void exclusive_scan_u32_pair(cudaStream_t st, const uint32_t* in0, uint32_t* out0, uint64_t n0,
                             const uint32_t* in1, uint32_t* out1, uint64_t n1, uint32_t* temp);
// The same scan in one launch (decoupled look-back, k_scan.cu).  temp holds
// scan1p_words(n) u32, 8-byte aligned, and must be zero when first used (its
// words are left ready for the next call).  err: optional flag word that gets
// SOIL_SCAN_ERR if a look-back wait runs out.
constexpr uint32_t SOIL_SCAN_ERR = 16u;
uint64_t scan1p_words(uint64_t n);
void exclusive_scan_1p(cudaStream_t st, const uint32_t* in, uint32_t* out, uint64_t n,
                       uint32_t* temp, uint32_t* err);

// ---- bins (k_bins.cu) -----------------------------------------------------
// cell[i] = cell_of(pos[first+i]) and counts[cell]++ for i in [0, n)
// pbc of locals [0, n) then cell_out[i] = their cell, counted (pbc + the sort's binning)
void launch_pbc_cells(cudaStream_t st, uint64_t n, const AtomCols& c, const Geom& g,
                      const double bvel[3], const Grid& gr, uint32_t* cell_out, uint32_t* counts);
// initial_integration (after the previous step's final one when fuse_final)
// and pbc of the locals in one pass, for a step that rebuilds for certain in a
// fully periodic box; with cell_out, also the sort's cells and counts (as
// launch_pbc_cells)
void launch_initial_pbc(cudaStream_t st, uint64_t n, const AtomCols& c, double dt,
                        bool fuse_final, bool zero_force, const Geom& g, const double bvel[3],
                        const Grid& gr, uint32_t* cell_out, uint32_t* counts);
// n_dev (optional, here and below): the count is min(n, *n_dev), read on the
// device (n an upper bound), for launches queued before the host knows it.
void launch_cells(cudaStream_t st, uint64_t first, uint64_t n, const AtomCols& c, const Grid& gr,
                  uint32_t* cell_out, uint32_t* counts, const uint32_t* n_dev = nullptr);
// counts[cell[i]]++ for i in [0, n) (cells already known)
void launch_count_cells(cudaStream_t st, uint64_t n, const uint32_t* cell, uint32_t* counts);
// out[cursor[cell[i]]++] = i (unordered within a cell)
void launch_scatter(cudaStream_t st, uint64_t n, const uint32_t* cell, uint32_t* cursor,
                    uint32_t* out);
// out[start[c] + --counts[c]] = i for c = cell[i] (unordered within a cell);
// leaves every count at zero
void launch_scatter_consume(cudaStream_t st, uint64_t n, const uint32_t* cell,
                            const uint32_t* start, uint32_t* counts, uint32_t* out,
                            const uint32_t* n_dev = nullptr);
// cell_out[i] = local_cell[i] (i < nlocal) or the cell of atom i, counted,
// i in [0, n)
void launch_cells_reuse(cudaStream_t st, uint64_t nlocal, uint64_t n, const AtomCols& c,
                        const Grid& gr, const uint32_t* local_cell, uint32_t* cell_out,
                        uint32_t* counts, const uint32_t* n_dev = nullptr);
// The neighbor build's bin order (out = sorted atoms) just after a spatial
// sort on the same grid: local i of cell c at start[c] + i - sort_start[c],
// then c's ghosts [nl, n) in ascending order after its locals.  counts: the
// cells' local + ghost counts (the ghosts' part is consumed); tmp: scratch of
// the atoms' size.  Returns true when counts[0, nc) were put back to zero
// (there were ghost slots to rank).
bool launch_place_bins(cudaStream_t st, uint64_t nl, uint64_t n, uint64_t nc,
                       const uint32_t* n_dev, const uint32_t* cell, const uint32_t* start,
                       const uint32_t* sort_start, uint32_t* counts, uint32_t* tmp,
                       uint32_t* out);
// sort every segment [start[s], start[s+1]) ascending -> stable counting sort
void launch_segsort(cudaStream_t st, uint64_t nseg, const uint32_t* start, uint32_t* items);
// the same, and split[s] = entries of segment s below s (transposed lists)
struct FillGuard;
void launch_segsort_split(cudaStream_t st, uint64_t nseg, const uint32_t* start, uint32_t* items,
                          uint32_t* split, const FillGuard* g = nullptr);
// split[s] alone, for segments already sorted
void launch_in_split(cudaStream_t st, uint64_t nseg, const uint32_t* start, const uint32_t* items,
                     uint32_t* split);
// dst[k] = src[perm[k]] for every column, k in [0, n)
// cell_out (optional): cell_out[k] = cell_in[perm[k]] in the same pass.
void launch_perm_gather(cudaStream_t st, uint64_t n, const uint32_t* perm, const AtomCols& src,
                        const AtomCols& dst, bool forces = true, const uint32_t* cell_in = nullptr,
                        uint32_t* cell_out = nullptr);
// flags->not_identity |= any perm[k] != k
void launch_identity_check(cudaStream_t st, uint64_t n, const uint32_t* perm, DevFlags* flags);
// out[k] = cell[perm[k]]
// Slot rows (max tags, max*width payload values per atom) of the n locals
// gathered through perm (dst row r = src row perm[r]).
void launch_slot_gather(cudaStream_t st, uint64_t n, const uint32_t* perm, uint32_t max,
                        uint32_t width, const uint32_t* src_tag, const double* src_val,
                        uint32_t* dst_tag, double* dst_val);
void launch_permute_u32(cudaStream_t st, uint64_t n, const uint32_t* perm, const uint32_t* in,
                        uint32_t* out);
// inverse[sorted[m]] = m and the sorted records sp[m] = {x, y, z, cutoff}
// (plus the FP32 grid-relative copy spf when spf != nullptr); atom_in_w (for
// a uniform cutoff, whose test reads no radius) stores sorted[m]'s bits in
// place of the cutoff; clear (when given, and n > 0) gets its candidates,
// rechecked and error words zeroed
void launch_sorted_views(cudaStream_t st, uint64_t n, const uint32_t* sorted, const AtomCols& c,
                         uint32_t* atom_sorted_idx, double4* sp, float4* spf,
                         const double origin[3], const BuildPos& bp = BuildPos{},
                         const uint32_t* n_dev = nullptr, bool atom_in_w = false,
                         DevFlags* clear = nullptr);

// ---- ghosts (k_ghost.cu) --------------------------------------------------
struct BorderDim {
    int dim;
    int triclinic;
    Geom geom;
    double thresh_lo;  // orthogonal: lo_face + gc;   triclinic: lo_face + cut_l
    double thresh_hi;  // orthogonal: hi_face - gc;   triclinic: hi_face - cut_l
    double shift[2][3];
    double vshift[2][3];
    int swap_id[2];
};
// Border state words of one borders pass (device memory, read back once):
//   [0..3] scan_end of dim d, [4..6] lo-swap totals, [7..9] hi-swap totals,
//   [10] overflow flag, [16 + k] image count of chain category k (k < 26),
//   [42] all images.
constexpr int kBorderStateWords = 48;
constexpr int kBorderCats = 26;
constexpr int kBorderTotals = 16;

// Geometry of one borders pass: face thresholds per dim, image shifts per
// swap id (2*dim + side, side 0 = the lo swap).
struct BorderPass {
    Geom geom;
    int triclinic;
    double lo[3], hi[3];
    double shift[kNumSwaps][3];
    double vshift[kNumSwaps][3];
};
// Chain categories of ghost images, in the order borders creates them
// (border_cats in k_ghost.cu): the face bits a root needs for category k,
// its swap chain, the parent category (-1: the root), the categories in
// reverse-fold order and the contiguous category range of every swap.
struct BorderCats {
    // per combination of the six face bits: the categories a root with those
    // bits belongs to (bit k), and the same set by fold position (bit f for
    // category fold[f]); set by finish_border_cats
    uint32_t member[64];
    uint32_t member_fold[64];
    uint8_t need[kBorderCats];
    uint8_t len[kBorderCats];
    uint8_t sw[kBorderCats][3];
    int8_t parent[kBorderCats];
    uint8_t swap_of[kBorderCats];
    uint8_t fold[kBorderCats];
    uint8_t swap_first[kNumSwaps];
    uint8_t swap_ncat[kNumSwaps];
};
const BorderCats& border_cats();
// Fill the member masks of a category table from its needs and fold order.
void finish_border_cats(BorderCats& t);
// The categories with every chain through a swap outside periodic_swaps (bit
// s: swap s has a periodic neighbor) made empty: they never match a root.
BorderCats border_cats_masked(unsigned periodic_swaps);
BorderPass border_pass(const BorderDim bds[3]);
struct SendPtrs {
    uint32_t* p[kNumSwaps];
};
// borders + the reverse-comm fold program in three launches: face bits and
// per-warp category counts of the locals, a scan per category, then every
// image written from its root.  bs must be zero; ghosts beyond `cap` set
// bs[10].  offs holds (kBorderCats + 1) * nw words and counts that plus
// (kBorderCats + 1) * ceil(nw / 8192) (nw = ceil(nlocal / 32)).
// cats: border_cats(), or border_cats_masked() for axes without periodicity.
// host_bs (optional, host memory mapped for the device): the kernels also
// write bs[0, 11) there, so no copy is needed after them.
void launch_borders(cudaStream_t st, uint64_t nlocal, uint64_t cap, const AtomCols& c,
                    const BorderCats& cats, const BorderPass& bp, uint8_t* face, uint32_t* counts,
                    uint32_t* offs,
                    uint32_t* bs, uint32_t* ghost_root, uint32_t* ghost_chain,
                    const SendPtrs& send, uint32_t* fold_start, uint32_t* fold_list,
                    uint32_t* host_bs = nullptr);
// forward_comm: every ghost from its root local atom through its swap chain
void launch_forward(cudaStream_t st, uint64_t nlocal, uint64_t nghost, const AtomCols& c,
                    const uint32_t* ghost_root, const uint32_t* ghost_chain, const SwapConst& sc,
                    const int* fwd_planes, int nfwd, bool zero_force);
// reverse_send_force: F[origin[g]] += F[g] (+ #[reverse] planes) over every
// root's image tree in fold order
void launch_reverse_fold(cudaStream_t st, uint64_t nlocal, const uint32_t* start,
                         const uint32_t* list, const AtomCols& c, const int* rev_planes, int nrev);
// The same fold over the roots that have images only: roots[0 .. *count)
// (count read on the device, at most max_roots)
void launch_reverse_fold_roots(cudaStream_t st, uint64_t nlocal, uint64_t max_roots,
                               const uint32_t* count, const uint32_t* roots,
                               const uint32_t* start, const uint32_t* list, const AtomCols& c,
                               const int* rev_planes, int nrev);
// flag[t] = local t has images (fold_start[t + 1] != fold_start[t]), t < nlocal
void launch_fold_root_flags(cudaStream_t st, uint64_t nlocal, const uint32_t* fold_start,
                            uint32_t* flag);

// ---- neighbor (k_neighbor.cu) ---------------------------------------------
struct PairParams {
    const uint32_t* atom_cell;
    const uint32_t* atom_sorted_idx;
    const uint32_t* bin_start;
    const uint32_t* sorted_atoms;
    const double4* sp;    // sorted {x, y, z, cutoff_radius}
    const float4* spf;    // FP32 grid-relative {x, y, z, cutoff_radius} (FP32 filter)
    const int32_t* stencil;  // runs of consecutive stencil cells: (offset, cells) pairs
    int nstencil;            // runs
    uint32_t ncells;      // bin_total_cells: stencil cells outside it are skipped and flagged
    uint64_t nlocal;
    int has_self;
    int newton;
    int uniform;
    int filter;
    int row_slots;        // K: row entries kept by pass 1 per atom
    double cut_sq;        // uniform: cached_uniform_cutoff_sq
    double sf_sq;         // skin_fraction^2
    double sf;            // skin_fraction
    float eps32;          // FP32 margin
    // The transposed lists built with the pairs (NULL: not here): pass 1
    // counts each row entry into in_count[partner]; pass 2 places row i in
    // every partner's list at in_start[partner] + (its count, consumed).
    uint32_t* in_count;
    const uint32_t* in_start;
    uint32_t* in_list;
    int pre_ranges;  // row_scan_pre for stencils of few runs (SOIL_PAIRS_PRE, default on)
};
// Pass 1: row lengths into rowcount[], the first K entries of each row into
// slots[i*K ...]; filter statistics into flags.
void launch_pair_count(cudaStream_t st, const PairParams& p, uint32_t* rowcount, uint32_t* slots,
                       DevFlags* flags);
// The stencil of a row as contiguous cell runs, in scan order: the own cell
// first (when the stencil holds it), then the stencil offsets merged into
// runs of consecutive cells.  A run of consecutive cells is a contiguous
// range of sorted slots, for one row and for a tile of rows alike.
// For staging, segments of consecutive cells merge into runs (the own cell
// with a following +1 segment).
constexpr int kMaxPairSegs = 24;
struct PairSegs {
    int n;                    // segments, own cell included
    int own;                  // 1: segment 0 is the own cell
    int32_t off[kMaxPairSegs];
    int32_t len[kMaxPairSegs];
    int32_t run[kMaxPairSegs];  // staging run of each segment
    int nrun;
    int32_t roff[kMaxPairSegs];
    int32_t rlen[kMaxPairSegs];
};
// Pass 1 with every warp's candidate records staged in shared memory by bulk
// copy (cp.async.bulk); tiles whose runs do not fit use the global-load scan.
// Same outputs as launch_pair_count.  flags->error bit 8: a staging wait ran out.
void launch_pair_count_staged(cudaStream_t st, const PairParams& p, const PairSegs& sg,
                              uint32_t* rowcount, uint32_t* slots, DevFlags* flags);
constexpr uint32_t SOIL_PAIRS_ERR_STAGING = 8u;
// A pass launched before the host has read the pair total runs only when the
// total fits its arrays: *total + 1 <= cap, and err[0] (DevFlags::error) and
// err[1] (DevFlags::fault) are clear.  Every thread reads the same words, so
// a launch runs whole or not at all.  A default guard (null total) is open.
// Pass 2 can also hand the host what it waits for (pub_total != null): the
// first thread copies *total to *pub_total and *flags to *pub_flags (host
// memory mapped for the device), whether or not the guard lets it run.
struct FillGuard {
    const uint32_t* total = nullptr;
    uint64_t cap = 0;
    const uint32_t* err = nullptr;
    uint32_t* pub_total = nullptr;
    const DevFlags* flags = nullptr;
    DevFlags* pub_flags = nullptr;
};
__device__ __forceinline__ bool guard_open(const FillGuard& g) {
    if (!g.total) return true;
    return (uint64_t)*g.total + 1 <= g.cap && g.err[0] == 0u && g.err[1] == 0u;
}
__device__ __forceinline__ void guard_publish(const FillGuard& g) {
    if (g.pub_total && blockIdx.x == 0 && threadIdx.x == 0) {
        *g.pub_total = *g.total;
        *g.pub_flags = *g.flags;
    }
}
// Pass 2: rows into neighbor_indices at offsets[] (rows longer than K re-derived).
void launch_pair_fill(cudaStream_t st, const PairParams& p, const uint32_t* rowcount,
                      const uint32_t* slots, const uint32_t* offsets, uint32_t* indices,
                      const FillGuard& g = FillGuard{});
// incoming (transposed) lists: for each atom j, the rows i with j in row(i)
void launch_in_count(cudaStream_t st, uint64_t nlocal, const uint32_t* offsets,
                     const uint32_t* indices, uint32_t* incount);
void launch_in_scatter(cudaStream_t st, uint64_t nlocal, const uint32_t* offsets,
                       const uint32_t* indices, uint32_t* cursor, uint32_t* in_list);

// ---- force (k_force.cu) ---------------------------------------------------
// Grouped partner sequences of the built-in consumer.  Atom a's sequence is
// its contributions in the reference's force-sum order (in-list rows below
// a, a's own row, in-list rows above a; ghosts only receive with newton).
// Root t's group is t's sequence, then those of its ghost images in fold
// order (fold_start / fold_list of the last border pass).
struct SeqArgs {
    uint64_t nlocal, ntotal;
    int newton;
    const uint32_t* offsets;
    const uint32_t* indices;
    const uint32_t* in_start;
    const uint32_t* in_list;
    const uint32_t* fold_start;
    const uint32_t* fold_list;
};
// cnt[a] = length of a's sequence (a < ntotal); grp[t] = length of t's group
void launch_seq_count(cudaStream_t st, const SeqArgs& q, uint32_t* cnt, uint32_t* grp);
// seq[grp_start[t] ...] = t's group; owner[k] = (t & 31) | item << 5 (item 0:
// the root, item j: its j-th image).  Roots have at most 7 images.
void launch_seq_fill(cudaStream_t st, const SeqArgs& q, const uint32_t* grp_start, uint32_t* seq,
                     uint8_t* owner);
// The grouped sequences and consumer constants of one system.
struct ForceSeq {
    const double* rad;
    double K;
    uint64_t nlocal;
    const uint32_t* grp_start;  // nlocal + 1
    const uint32_t* cnt;        // per atom
    const uint32_t* seq;
    const uint8_t* owner;
    const uint32_t* fold_start;
    const uint32_t* fold_list;
    const double* pk;  // packed (x, y, z, r) records, current; NULL: the columns
};
struct ForceArgs {
    AtomCols c;
    ForceSeq q;
    PlaneList rev;  // #[reverse] planes folded with the forces
};
// Kernels of the built-in consumer (SOIL_FORCE): the per-atom gather over the
// CSR and its transpose with a separate reverse pass (GATHER); one thread per
// root walking its and its images' transposed lists and rows, with the fold
// (CSR); or a kernel over grouped sequences built at each rebuild, with the
// fold: warp tiles of 32 roots with 4 or 2 rows of 32 entries per chunk
// (TILES4, TILES2), or one thread per root walking its group (WALK).
enum {
    SOIL_FORCE_GATHER = 0,
    SOIL_FORCE_TILES4 = 1,
    SOIL_FORCE_TILES2 = 2,
    SOIL_FORCE_WALK = 3,
    SOIL_FORCE_CSR = 4
};
constexpr int kDefaultForce = SOIL_FORCE_CSR;  // when SOIL_FORCE is unset
// The consumer walking each root's transposed list and CSR row directly
// (one thread per root, its images after it, then the fold): no grouped
// sequences are built.
struct ForceCsr {
    const double* rad;
    double K;
    uint64_t nlocal;
    int newton;
    const uint32_t* offsets;
    const uint32_t* indices;
    const uint32_t* in_start;
    const uint32_t* in_list;
    const uint32_t* in_split;  // per atom: in-list entries below it
    const uint32_t* fold_start;
    const uint32_t* fold_list;
    // Roots by work inside each block of kBlock roots (NULL: index order):
    // thread k of the block that takes roots [b, b + kBlock) walks
    // order[b + k].  Threads of a warp then walk groups of similar length.
    const uint32_t* order;
    const double* pk;  // packed (x, y, z, r) records, current; NULL: the columns
};
void launch_force_csr(cudaStream_t st, const ForceCsr& q, const AtomCols& c, const PlaneList& rev,
                      bool fold);
// order[b + k] for every block of kBlock roots: the block's roots sorted by
// their entry count (their own and their images' in-list and row lengths),
// ties in index order.
void launch_root_order(cudaStream_t st, const ForceCsr& q, uint32_t* order);
int force_variant();  // from SOIL_FORCE (default chosen by measurement)
// The built-in consumer over the grouped sequences: F of every local and
// ghost is overwritten; with fold, ghost forces (and the #[reverse] planes)
// are then folded into their roots as reverse comm does.
void launch_force_seq(cudaStream_t st, const ForceArgs& p, bool fold, int variant);

// ---- device-resident steps (k_steps.cu) --------------------------------------
// Grid barrier words (count must be 0 when a launch starts).
struct GridBar {
    unsigned count;
    unsigned gen;
};
constexpr uint32_t SOIL_STEPS_ERR_BARRIER = 4u;  // flags->error: a barrier wait ran out
struct StepsArgs {
    AtomCols c;
    uint64_t nlocal;
    double dt;
    int zero_force;    // zero the locals' forces in the integration pass
    int first_fused;   // the first step's pass also applies the pending final half-kick
    CheckArgs ck;      // the displacement check (every step)
    FwdArgs fw;        // forward comm of every step
    ForceArgs fa;      // the grouped consumer (consumer != 0, mode 0 / 1)
    ForceCsr fc;       // the CSR walk (consumer != 0, mode 2)
    int walk;          // consumer mode: 0 warp tiles, 1 grouped walk, 2 CSR walk
    uint64_t max_steps;
    GridBar* bar;
    DevFlags* flags;   // flags->rebuild is set when a check trips
    uint32_t* out;     // out[0]: steps completed; out[1]: 1 if the next step's check tripped
    uint32_t* trip;    // 3 check-flag slots, zero at launch
};
// Cooperative grid for k_steps (consumer: 0 none, 1 grouped, 2 grouped + fold).
int steps_grid(int consumer, int walk, bool pk, uint64_t nlocal, int* grid);
cudaError_t launch_steps(cudaStream_t st, const StepsArgs& a, int consumer, int walk, bool pk,
                         int grid);

void launch_harmonic(cudaStream_t st, uint64_t nlocal, uint64_t ntotal, const AtomCols& c,
                     const double* radius, double k, int newton, const uint32_t* offsets,
                     const uint32_t* indices, const uint32_t* in_start, const uint32_t* in_list);

}  // namespace soil
