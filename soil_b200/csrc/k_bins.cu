// k_bins.cu — binning and the stable counting sort used by both the spatial
// sort (sort_atoms_by_bin, neighbor.rs:834-997) and the neighbor build's bin
// fill (bin_neighbor_list, neighbor.rs:1046-1125).
//
// The reference's counting sort is stable: inside a cell atoms keep
// ascending index.  The device version counts with warp-aggregated atomics
// (__match_any_sync on the cell id, one atomicAdd per distinct cell per
// warp), scans, scatters with the same aggregated atomics (order inside a cell
// is then arbitrary), and restores the stable order by sorting each cell's
// segment by atom index.  Cells hold ~2 atoms on average, so that last pass
// is a short insertion sort per cell.
#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

__global__ void __launch_bounds__(kBlock) k_cells(uint64_t first, uint64_t n, AtomCols c, Grid gr,
                                                  uint32_t* cell_out, uint32_t* counts,
                                                  const uint32_t* n_dev) {
    if (n_dev) {  // the count known only on the device (an upper bound in n)
        const uint64_t d = *n_dev;
        n = d < n ? d : n;
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        uint32_t cell = 0;
        if (valid) {
            const uint64_t a = first + i;
            cell = cell_of(gr, c.x[a], c.y[a], c.z[a]);
            cell_out[i] = cell;
        }
        aggregated_count(counts, cell, valid);
    }
}

// pbc of the locals and the sort's cells in one pass: each local is wrapped
// (pbc_atom) and its new position binned and counted.
__global__ void __launch_bounds__(kBlock) k_pbc_cells(uint64_t n, AtomCols c, Geom g, double bv0,
                                                      double bv1, double bv2, Grid gr,
                                                      uint32_t* cell_out, uint32_t* counts) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        uint32_t cell = 0;
        if (valid) {
            double x, y, z;
            pbc_atom(c, i, g, bv0, bv1, bv2, x, y, z);
            cell = cell_of(gr, x, y, z);
            cell_out[i] = cell;
        }
        aggregated_count(counts, cell, valid);
    }
}

// The integration pass of a step that rebuilds for certain, in a fully
// periodic box: initial_integration (with the previous step's final half-kick
// when FUSE_FINAL) and pbc of the new position in registers, every column
// stored once; with CELLS the wrapped position binned and counted for the
// sort.  Same arithmetic as initial_atom followed by pbc_atom.
template <bool FUSE_FINAL, bool CELLS>
__global__ void __launch_bounds__(kBlock) k_initial_pbc(uint64_t n, AtomCols c, double dt,
                                                        int zero_force, Geom g, double bv0,
                                                        double bv1, double bv2, Grid gr,
                                                        uint32_t* cell_out, uint32_t* counts) {
    pdl_wait();  // launched with pdl_launch
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t cap = c.cap;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        uint32_t cell = 0;
        if (valid) {
            const double h = 0.5 * dt * c.inv_mass[i];
            const double fx = c.fx[i], fy = c.fy[i], fz = c.fz[i];
            double vx = c.vx[i], vy = c.vy[i], vz = c.vz[i];
            double x = c.x[i], y = c.y[i], z = c.z[i];
            int32_t m0 = c.img[i], m1 = c.img[cap + i], m2 = c.img[2 * cap + i];
            initial_regs(h, dt, FUSE_FINAL, fx, fy, fz, vx, vy, vz, x, y, z);
            pbc_core(g, x, y, z, m0, m1, m2, [&](double sg) {
                vx = vx - sg * bv0;
                vy = vy - sg * bv1;
                vz = vz - sg * bv2;
            });
            c.vx[i] = vx;
            c.vy[i] = vy;
            c.vz[i] = vz;
            c.x[i] = x;
            c.y[i] = y;
            c.z[i] = z;
            c.img[i] = m0;
            c.img[cap + i] = m1;
            c.img[2 * cap + i] = m2;
            if (zero_force) {
                c.fx[i] = 0.0;
                c.fy[i] = 0.0;
                c.fz[i] = 0.0;
            }
            if (CELLS) {
                cell = cell_of(gr, x, y, z);
                cell_out[i] = cell;
            }
        }
        if (CELLS) aggregated_count(counts, cell, valid);
    }
}

template <bool FUSE_FINAL, bool CELLS>
static void initial_pbc_t(cudaStream_t st, uint64_t n, const AtomCols& c, double dt,
                          bool zero_force, const Geom& g, const double bvel[3], const Grid& gr,
                          uint32_t* cell_out, uint32_t* counts) {
    pdl_launch(k_initial_pbc<FUSE_FINAL, CELLS>, grid_wave<k_initial_pbc<FUSE_FINAL, CELLS>>(n), kBlock, 0, st, n, c, dt, zero_force ? 1 : 0, g, bvel[0], bvel[1],
                                             bvel[2], gr, cell_out, counts);
}

void launch_initial_pbc(cudaStream_t st, uint64_t n, const AtomCols& c, double dt,
                        bool fuse_final, bool zero_force, const Geom& g, const double bvel[3],
                        const Grid& gr, uint32_t* cell_out, uint32_t* counts) {
    if (n == 0) return;
    note_launch();
    if (fuse_final) {
        if (cell_out) initial_pbc_t<true, true>(st, n, c, dt, zero_force, g, bvel, gr, cell_out, counts);
        else initial_pbc_t<true, false>(st, n, c, dt, zero_force, g, bvel, gr, cell_out, counts);
    } else {
        if (cell_out) initial_pbc_t<false, true>(st, n, c, dt, zero_force, g, bvel, gr, cell_out, counts);
        else initial_pbc_t<false, false>(st, n, c, dt, zero_force, g, bvel, gr, cell_out, counts);
    }
}

void launch_pbc_cells(cudaStream_t st, uint64_t n, const AtomCols& c, const Geom& g,
                      const double bvel[3], const Grid& gr, uint32_t* cell_out, uint32_t* counts) {
    if (n == 0) return;
    note_launch();
    k_pbc_cells<<<grid_wave<k_pbc_cells>(n), kBlock, 0, st>>>(n, c, g, bvel[0], bvel[1], bvel[2],
                                                              gr, cell_out, counts);
}

void launch_cells(cudaStream_t st, uint64_t first, uint64_t n, const AtomCols& c, const Grid& gr,
                  uint32_t* cell_out, uint32_t* counts, const uint32_t* n_dev) {
    if (n == 0) return;
    note_launch();
    k_cells<<<grid_wave<k_cells>(n), kBlock, 0, st>>>(first, n, c, gr, cell_out, counts, n_dev);
}

__global__ void __launch_bounds__(kBlock) k_count_cells(uint64_t n, const uint32_t* cell,
                                                        uint32_t* counts) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        aggregated_count(counts, valid ? cell[i] : 0u, valid);
    }
}

void launch_count_cells(cudaStream_t st, uint64_t n, const uint32_t* cell, uint32_t* counts) {
    if (n == 0) return;
    note_launch();
    k_count_cells<<<grid_wave<k_count_cells>(n), kBlock, 0, st>>>(n, cell, counts);
}

__global__ void __launch_bounds__(kBlock) k_scatter(uint64_t n, const uint32_t* cell,
                                                    uint32_t* cursor, uint32_t* out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? cell[i] : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (valid && lane == leader) base = atomicAdd(&cursor[key], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (valid) out[base + __popc(peers & lanemask_lt())] = (uint32_t)i;
    }
}

void launch_scatter(cudaStream_t st, uint64_t n, const uint32_t* cell, uint32_t* cursor,
                    uint32_t* out) {
    if (n == 0) return;
    note_launch();
    k_scatter<<<grid_wave<k_scatter>(n), kBlock, 0, st>>>(n, cell, cursor, out);
}

// The scatter that consumes the counts: out[start[c] + --counts[c]] = i
// (warp-aggregated), so every count is zero again afterwards and the next
// counting pass needs no clearing; the order inside a cell is restored by
// the segment sort that follows.
__global__ void __launch_bounds__(kBlock) k_scatter_consume(uint64_t n, const uint32_t* cell,
                                                            const uint32_t* start,
                                                            uint32_t* counts, uint32_t* out,
                                                            const uint32_t* n_dev) {
    pdl_wait();  // launched with pdl_launch
    if (n_dev) {  // the count known only on the device (an upper bound in n)
        const uint64_t d = *n_dev;
        n = d < n ? d : n;
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        const uint32_t key = valid ? cell[i] : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        const uint32_t k = (uint32_t)__popc(peers);
        uint32_t top = 0;  // the count before this warp's claim
        if (valid && lane == leader) top = atomicSub(&counts[key], k);
        top = __shfl_sync(0xffffffffu, top, leader);
        if (valid) out[start[key] + (top - k) + __popc(peers & lanemask_lt())] = (uint32_t)i;
    }
}

void launch_scatter_consume(cudaStream_t st, uint64_t n, const uint32_t* cell,
                            const uint32_t* start, uint32_t* counts, uint32_t* out,
                            const uint32_t* n_dev) {
    if (n == 0) return;
    note_launch();
    pdl_launch(k_scatter_consume, grid_wave<k_scatter_consume>(n), kBlock, 0, st, n, cell, start, counts,
                                                                          out, n_dev);
}

// The neighbor build's cells in one pass: the locals' cells from the sort
// (local < nlocal), the others' from their positions; all counted.
__global__ void __launch_bounds__(kBlock) k_cells_reuse(uint64_t nlocal, uint64_t n, AtomCols c,
                                                        Grid gr, const uint32_t* local_cell,
                                                        uint32_t* cell_out, uint32_t* counts,
                                                        const uint32_t* n_dev) {
    pdl_wait();  // launched with pdl_launch
    if (n_dev) {  // the count known only on the device (an upper bound in n)
        const uint64_t d = *n_dev;
        n = d < n ? d : n;
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        uint32_t cell = 0;
        if (valid) {
            cell = i < nlocal ? local_cell[i] : cell_of(gr, c.x[i], c.y[i], c.z[i]);
            cell_out[i] = cell;
        }
        aggregated_count(counts, cell, valid);
    }
}

void launch_cells_reuse(cudaStream_t st, uint64_t nlocal, uint64_t n, const AtomCols& c,
                        const Grid& gr, const uint32_t* local_cell, uint32_t* cell_out,
                        uint32_t* counts, const uint32_t* n_dev) {
    if (n == 0) return;
    note_launch();
    pdl_launch(k_cells_reuse, grid_wave<k_cells_reuse>(n), kBlock, 0, st, nlocal, n, c, gr, local_cell,
                                                                  cell_out, counts, n_dev);
}

// The neighbor build's bins right after a spatial sort of the same grid:
// the locals are already in cell order (local i is entry i - sort_start[c]
// of its cell c), so they take their slots directly, in front of their
// cell's ghosts; only the ghosts are scattered and ranked.
// One pass over all atoms: local i (its cell's locals are consecutive in
// bin order already) straight to its slot; ghost g of cell c into the ghost
// part of c's slots (after its locals), in no particular order: counts[c]
// still holds c's locals and ghosts, and only ghosts take from it.
__global__ void __launch_bounds__(kBlock) k_place_bins(uint64_t nl, uint64_t n,
                                                       const uint32_t* n_dev,
                                                       const uint32_t* cell,
                                                       const uint32_t* start,
                                                       const uint32_t* sort_start,
                                                       uint32_t* counts, uint32_t* tmp,
                                                       uint32_t* out) {
    pdl_wait();  // launched with pdl_launch
    if (n_dev) {
        const uint64_t d = *n_dev;
        n = d < n ? d : n;
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = cell[i];
        if (i < nl) out[start[c] + ((uint32_t)i - sort_start[c])] = (uint32_t)i;
        else tmp[start[c] + atomicSub(&counts[c], 1u) - 1u] = (uint32_t)i;
    }
}

// Each ghost at its rank among its cell's ghosts (ascending index).
// The cells' counts (read by nothing after k_place_bins) go back to zero on
// the way, for the next counting pass.
__global__ void __launch_bounds__(kBlock) k_ghost_rank(uint64_t nl, uint64_t n,
                                                       const uint32_t* n_dev,
                                                       const uint32_t* cell,
                                                       const uint32_t* start,
                                                       const uint32_t* sort_start,
                                                       const uint32_t* tmp, uint32_t* out,
                                                       uint32_t* counts, uint64_t nc) {
    pdl_wait();  // launched with pdl_launch
    if (n_dev) {
        const uint64_t d = *n_dev;
        n = d < n ? d : n;
    }
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < nc;
         c += (uint64_t)gridDim.x * blockDim.x)
        counts[c] = 0u;
    for (uint64_t g = nl + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = cell[g];
        const uint32_t gb = start[c] + (sort_start[c + 1] - sort_start[c]), ge = start[c + 1];
        uint32_t rank = 0;
        for (uint32_t j = gb; j < ge; ++j) rank += tmp[j] < (uint32_t)g;
        out[gb + rank] = (uint32_t)g;
    }
}

bool launch_place_bins(cudaStream_t st, uint64_t nl, uint64_t n, uint64_t nc,
                       const uint32_t* n_dev, const uint32_t* cell, const uint32_t* start,
                       const uint32_t* sort_start, uint32_t* counts, uint32_t* tmp,
                       uint32_t* out) {
    if (n == 0) return false;
    note_launch();
    pdl_launch(k_place_bins, grid_wave<k_place_bins>(n), kBlock, 0, st, nl, n, n_dev, cell, start,
                                                                 sort_start, counts, tmp, out);
    if (n == nl) return false;
    note_launch();
    const uint64_t rank_items = n - nl > nc ? n - nl : nc;  // ghosts, or cells to clear
    pdl_launch(k_ghost_rank, grid_wave<k_ghost_rank>(rank_items), kBlock, 0, st, 
        nl, n, n_dev, cell, start, sort_start, tmp, out, counts, nc);
    return true;
}

// One thread per segment, sorted in place (in registers for up to 8 items,
// sort_segment).  SPLIT: split[s] = the items of segment s below s.  (Staging
// each warp's 32 segments through shared memory, read and written back
// coalesced, measured slower: 0.450 against 0.441 ms per C3 step.)
template <bool SPLIT>
__device__ __forceinline__ void segsort_lanes(uint64_t nseg, const uint32_t* start,
                                              uint32_t* items, uint32_t* split) {
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nseg;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t below = sort_segment(items, start[s], start[s + 1], (uint32_t)s);
        if (SPLIT) split[s] = below;
    }
}

// Restore the stable (ascending index) order inside every segment.
__global__ void __launch_bounds__(kBlock) k_segsort(uint64_t nseg, const uint32_t* start,
                                                    uint32_t* items) {
    pdl_wait();  // launched with pdl_launch
    segsort_lanes<false>(nseg, start, items, nullptr);
}

void launch_segsort(cudaStream_t st, uint64_t nseg, const uint32_t* start, uint32_t* items) {
    if (nseg == 0) return;
    note_launch();
    pdl_launch(k_segsort, grid_wave<k_segsort>(nseg), kBlock, 0, st, nseg, start, items);
}

// The transposed lists' sort: segment a (atom a's in-list) ascending, and
// split[a] = its entries below a (the rows summed before a's own row).
__global__ void __launch_bounds__(kBlock) k_segsort_split(uint64_t nseg, const uint32_t* start,
                                                          uint32_t* items, uint32_t* split,
                                                          FillGuard g) {
    pdl_wait();  // launched with pdl_launch
    if (!guard_open(g)) return;
    segsort_lanes<true>(nseg, start, items, split);
}

void launch_segsort_split(cudaStream_t st, uint64_t nseg, const uint32_t* start, uint32_t* items,
                          uint32_t* split, const FillGuard* g) {
    if (nseg == 0) return;
    note_launch();
    pdl_launch(k_segsort_split, grid_wave<k_segsort_split>(nseg), kBlock, 0, st, nseg, start,
               items, split, g ? *g : FillGuard{});
}

// split[a] of already sorted transposed lists
__global__ void __launch_bounds__(kBlock) k_in_split(uint64_t nseg, const uint32_t* start,
                                                     const uint32_t* items, uint32_t* split) {
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nseg;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = start[s], e = start[s + 1];
        uint32_t k = b;
        while (k < e && items[k] < (uint32_t)s) ++k;
        split[s] = k - b;
    }
}

void launch_in_split(cudaStream_t st, uint64_t nseg, const uint32_t* start, const uint32_t* items,
                     uint32_t* split) {
    if (nseg == 0) return;
    note_launch();
    k_in_split<<<grid_wave<k_in_split>(nseg), kBlock, 0, st>>>(nseg, start, items, split);
}

// Atom::apply_permutation + AtomDataRegistry::apply_permutation_all
// (atom.rs:479-490, 284-289): every column gathered through perm.
__global__ void __launch_bounds__(kBlock) k_perm_gather(uint64_t n, const uint32_t* perm,
                                                        AtomCols s, AtomCols d, int forces,
                                                        const uint32_t* cell_in,
                                                        uint32_t* cell_out) {
    pdl_wait();  // launched with pdl_launch
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = perm[k];
        perm_gather_atom(s, d, k, p, forces != 0);
        if (cell_out) cell_out[k] = cell_in[p];
    }
}

void launch_perm_gather(cudaStream_t st, uint64_t n, const uint32_t* perm, const AtomCols& src,
                        const AtomCols& dst, bool forces, const uint32_t* cell_in,
                        uint32_t* cell_out) {
    if (n == 0) return;
    note_launch();
    pdl_launch(k_perm_gather, grid_wave<k_perm_gather>(n), kBlock, 0, st, n, perm, src, dst, forces ? 1 : 0,
                                                                  cell_in, cell_out);
}

__global__ void __launch_bounds__(kBlock) k_identity(uint64_t n, const uint32_t* perm,
                                                     DevFlags* flags) {
    bool diff = false;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
         k += (uint64_t)gridDim.x * blockDim.x)
        diff |= perm[k] != (uint32_t)k;
    if (__ballot_sync(0xffffffffu, diff) && (threadIdx.x & 31) == 0)
        atomicOr(&flags->not_identity, 1u);
}

void launch_identity_check(cudaStream_t st, uint64_t n, const uint32_t* perm, DevFlags* flags) {
    if (n == 0) return;
    note_launch();
    k_identity<<<grid_wave<k_identity>(n), kBlock, 0, st>>>(n, perm, flags);
}

__global__ void __launch_bounds__(kBlock) k_permute_u32(uint64_t n, const uint32_t* perm,
                                                        const uint32_t* in, uint32_t* out) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
         k += (uint64_t)gridDim.x * blockDim.x)
        out[k] = in[perm[k]];
}

void launch_permute_u32(cudaStream_t st, uint64_t n, const uint32_t* perm, const uint32_t* in,
                        uint32_t* out) {
    if (n == 0) return;
    note_launch();
    k_permute_u32<<<grid_wave<k_permute_u32>(n), kBlock, 0, st>>>(n, perm, in, out);
}

// atom_sorted_idx and sorted_pos of bin_neighbor_list (neighbor.rs:1101-1125),
// as one record {x, y, z, cutoff_radius} per sorted slot, plus the FP32
// grid-relative copy the FP32 filter reads.
__global__ void __launch_bounds__(kBlock) k_sorted_views(uint64_t n, const uint32_t* sorted,
                                                         AtomCols c, uint32_t* asi, double4* sp,
                                                         float4* spf, double o0, double o1,
                                                         double o2, BuildPos bp,
                                                         const uint32_t* n_dev, int atom_in_w,
                                                         DevFlags* clear) {
    pdl_wait();  // launched with pdl_launch
    if (clear && blockIdx.x == 0 && threadIdx.x == 0) {  // the pair build's counters
        clear->candidates = 0;
        clear->rechecked = 0;
        clear->error = 0u;
    }
    if (n_dev) {  // the count known only on the device (an upper bound in n)
        const uint64_t d = *n_dev;
        n = d < n ? d : n;
    }
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < n;
         m += (uint64_t)gridDim.x * blockDim.x)
        sorted_view(c, m, sorted, asi, sp, spf, o0, o1, o2, bp, atom_in_w != 0);
}

void launch_sorted_views(cudaStream_t st, uint64_t n, const uint32_t* sorted, const AtomCols& c,
                         uint32_t* atom_sorted_idx, double4* sp, float4* spf,
                         const double origin[3], const BuildPos& bp, const uint32_t* n_dev,
                         bool atom_in_w, DevFlags* clear) {
    if (n == 0) return;
    note_launch();
    pdl_launch(k_sorted_views, grid_wave<k_sorted_views>(n), kBlock, 0, st, 
        n, sorted, c, atom_sorted_idx, sp, spf, origin[0], origin[1], origin[2], bp, n_dev,
        atom_in_w ? 1 : 0, clear);
}

}  // namespace soil
