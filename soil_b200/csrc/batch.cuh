// batch.cuh — device-side descriptors of the batched engine: many independent
// systems ("boxes") advanced together, each phase one kernel launch over all
// participating boxes.
//
// A launch covers a flattened element range split into segments, one per
// participating box (Span: the box of each segment, the segment's first
// flattened element, and the element offset inside the box — e.g. nlocal for
// a box's ghost range).  Blocks locate their segment once per chunk and then
// advance; every element runs the same per-element device function as the
// single-system kernels (device_ops.cuh), so a box's arithmetic is identical
// alone and batched.
#pragma once

#include "device_ops.cuh"

namespace soil {

constexpr int kMaxStencil = 96;  // stencil words per box: (offset, cells) runs

// Pointers of one box's arrays; changes only when the box's arrays are
// reallocated.  set[0]/set[1] are the two physical column sets; which one is
// current is a per-step value (the spatial sort gathers from one into the
// other).
struct BoxDev {
    AtomCols set[2];
    int radius_plane;  // registered plane holding the consumer's radius (-1: none)
    double shear_rate;  // streaming profile of the first shear step
    double yc;
    double* lbx;
    double* lby;
    double* lbz;
    uint32_t* sort_cell;
    uint32_t* sort_perm;
    uint32_t* sorted_local_cell;
    uint32_t* cell_counts;
    uint32_t* cell_start;
    uint32_t* cell_cursor;
    uint32_t* atom_cell;
    uint32_t* sorted_atoms;
    uint32_t* asi;
    uint32_t* rowcount;
    uint32_t* row_slots;
    uint32_t* offsets;
    uint32_t* indices;
    double4* sp;
    float4* spf;
    uint32_t* in_count;
    uint32_t* in_start;
    uint32_t* in_cursor;
    uint32_t* in_list;
    uint32_t* ghost_root;
    uint32_t* ghost_chain;
    uint32_t* send[kNumSwaps];
    uint8_t* face_flags;
    uint32_t* bcount;      // per-warp chain-category counts of borders
    uint32_t* boff;        // their offsets
    uint32_t* fold_start;
    uint32_t* fold_list;
    // grouped partner sequences of the built-in consumer (force_ops.cuh)
    uint32_t* seq_cnt;
    uint32_t* grp_cnt;
    uint32_t* grp_start;
    uint32_t* seq;
    uint8_t* seq_owner;
    uint64_t cap;  // atom capacity of both column sets
    PlaneList fwd, rev, zero;
};

// Per-step values of one box, rebuilt by the host every step.
struct BoxStep {
    uint64_t nlocal;
    uint64_t nghost;
    int cur;   // column set current before this step's spatial sort
    int post;  // column set current after it (== cur when no permutation applies)
    double dt;
    Geom geom;
    double bvel[3];
    Grid grid;
    uint32_t ncells;
    int32_t nstencil;
    int32_t stencil[kMaxStencil];
    int pre_ranges;  // the pair scan preloads its ranges
    int has_self;
    int newton;
    int uniform;
    int filter;
    double cut_sq;
    double sf_sq;
    double sf;
    float eps32;
    double thr_sq;
    double box[3];
    double ibox[3];
    double thresh_lo[3];
    double thresh_hi[3];
    SwapConst sc;
    double K;
    uint32_t max_tiles;
    int segs_ok;   // the stencil fits PairSegs: the pair count stages its records
    PairSegs segs;
};

struct Span {
    const uint32_t* box;    // box of each segment
    const uint64_t* start;  // first flattened element of each segment; start[nseg] = total
    const uint32_t* base;   // element offset inside the box
    const uint8_t* flag;    // per-segment switches (kernel specific)
    uint32_t nseg;
    uint64_t total;
};

struct BatchArgs {
    const BoxDev* dev;
    const BoxStep* step;
    DevFlags* flags;    // one per box
    uint32_t* bstate;   // kBorderStateWords per box
    uint32_t* totals;   // one per box (pair totals)
};

// Arrays a batched scan / zero / sort can target.
enum BatchArray {
    BA_CELLS = 0,     // cell_counts -> cell_start (+ cursor), segsort of sort_perm
    BA_NEIGH_CELLS,   // cell_counts -> cell_start (+ cursor), segsort of sorted_atoms
    BA_ROWS,          // rowcount -> offsets (total into totals[box])
    BA_IN,            // in_count -> in_start (+ cursor), segsort of in_list
    BA_GRP            // grp_cnt -> grp_start (grouped sequences)
};

// ---- launchers (k_batch.cu); every one enqueues a single kernel ------------
// integrate: flag bit0 check, bit1 fuse previous final, bit2 zero forces
void b_initial(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_final(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_profile(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_zero_forces(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_pbc(cudaStream_t st, const Span& sp, const BatchArgs& a);
// zero the counts of `which` over each segment's element range
void b_zero_counts(cudaStream_t st, const Span& sp, const BatchArgs& a, int which);
// cells of positions (sort: locals into sort_cell; neighbor: any range into atom_cell)
void b_cells(cudaStream_t st, const Span& sp, const BatchArgs& a, bool neighbor);
void b_copy_count_local_cells(cudaStream_t st, const Span& sp, const BatchArgs& a);
// one CTA per segment: exclusive scan of `which`, cursor copy, totals
void b_scan(cudaStream_t st, const Span& sp, const BatchArgs& a, int which);
void b_scatter(cudaStream_t st, const Span& sp, const BatchArgs& a, bool neighbor);
void b_segsort(cudaStream_t st, const Span& sp, const BatchArgs& a, int which);
void b_permute_cells(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_identity(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_perm_gather(cudaStream_t st, const Span& sp, const BatchArgs& a);
// borders + fold program (chain categories, see k_ghost.cu): element = warp
// tile of 32 locals of a box; the scan runs one CTA per (box, category)
void b_border_faces(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_border_cat_scan(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_border_images(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_forward(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_save_positions(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_sorted_views(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_pairs_rows(cudaStream_t st, const Span& sp, const BatchArgs& a);
// the pair count pass over warp tiles of 32 rows (element = tile of a box),
// candidate records staged in shared memory (pairs_staged.cuh)
void b_pairs_staged(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_pairs_fill(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_in_count(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_in_scatter(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_harmonic(cudaStream_t st, const Span& sp, const BatchArgs& a);
// grouped sequences: lengths over every atom (count) and the groups of the
// locals (fill, after a BA_GRP scan); the consumer over warp tiles of 32
// roots (element = tile of a box), folding images into roots with newton
void b_seq_count(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_seq_fill(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_force_grouped(cudaStream_t st, const Span& sp, const BatchArgs& a);
// the same consumer with one root per thread (element = local root)
void b_force_walk(cudaStream_t st, const Span& sp, const BatchArgs& a);
void b_reverse(cudaStream_t st, const Span& sp, const BatchArgs& a);

}  // namespace soil
