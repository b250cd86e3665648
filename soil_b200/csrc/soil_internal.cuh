// soil_internal.cuh — device/host shared definitions of the soil_b200 library.
//
// Device layout (structure of arrays, FP64 state):
//   atoms [0, nlocal) are local, [nlocal, nlocal+nghost) are periodic ghost
//   images appended by `borders` in the reference order.  Every per-atom
//   column is one or more planes of `acap` elements; column c of width w
//   occupies w consecutive planes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "soil_cuda.h"

namespace soil {

constexpr int kMaxCols = 16;      // registered AtomData columns per system
constexpr int kMaxPlanes = 48;    // f64 planes over all registered columns
constexpr int kNumSwaps = 6;      // one rank: (x,y,z) x (lo,hi)
constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// Device helpers shared by the kernels.  All arithmetic keeps the reference's
// operation order; the library is compiled with -fmad=false so a*b+c is never
// contracted, and fma() appears only where the reference calls mul_add.
// ---------------------------------------------------------------------------
__host__ __device__ inline int32_t sat_i32(double v) {
    // Rust `f64 as i32`: saturating, NaN -> 0
    if (v != v) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (int32_t)(-2147483647 - 1);
    return (int32_t)v;
}
__host__ __device__ inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

// Domain geometry needed on the device (Domain, domain.rs:105-142).
struct Geom {
    double lo[3];
    double size[3];
    double tilt[3];  // xy, xz, yz
    int triclinic;
};

// Domain::x2lamda, domain.rs:211-217
__device__ __forceinline__ void x2lamda(const Geom& g, double rx, double ry, double rz,
                                        double& lx, double& ly, double& lz) {
    const double xy = g.tilt[0], xz = g.tilt[1], yz = g.tilt[2];
    lz = (rz - g.lo[2]) / g.size[2];
    ly = (ry - g.lo[1] - yz * lz) / g.size[1];
    lx = (rx - g.lo[0] - xy * ly - xz * lz) / g.size[0];
}
// Domain::lamda2x, domain.rs:222-229
__device__ __forceinline__ void lamda2x(const Geom& g, double lx, double ly, double lz,
                                        double& rx, double& ry, double& rz) {
    const double xy = g.tilt[0], xz = g.tilt[1], yz = g.tilt[2];
    rx = g.lo[0] + g.size[0] * lx + xy * ly + xz * lz;
    ry = g.lo[1] + g.size[1] * ly + yz * lz;
    rz = g.lo[2] + g.size[2] * lz;
}

// Bin grid (Neighbor.bin_origin/bin_size/bin_count, neighbor.rs:311-495).
struct Grid {
    double origin[3];
    double inv_bs[3];  // 1.0 / bin_size, computed on the host as the reference does
    int32_t n[3];
    Geom geom;
};

// Cell of a position: sort_atoms_by_bin (neighbor.rs:912-923) and
// bin_neighbor_list (neighbor.rs:1070-1083) use the same formula.
__device__ __forceinline__ uint32_t cell_of(const Grid& gr, double px, double py, double pz) {
    double p0 = px, p1 = py, p2 = pz;
    if (gr.geom.triclinic) x2lamda(gr.geom, px, py, pz, p0, p1, p2);
    const int32_t nx = gr.n[0], ny = gr.n[1], nz = gr.n[2];
    int32_t cx = clampi(sat_i32(floor((p0 - gr.origin[0]) * gr.inv_bs[0])), 0, nx - 1);
    int32_t cy = clampi(sat_i32(floor((p1 - gr.origin[1]) * gr.inv_bs[1])), 0, ny - 1);
    int32_t cz = clampi(sat_i32(floor((p2 - gr.origin[2]) * gr.inv_bs[2])), 0, nz - 1);
    return (uint32_t)(cx * ny * nz + cy * nz + cz);
}

// Pointers of all per-atom columns (base + registered planes).
struct AtomCols {
    double* x;
    double* y;
    double* z;
    double* vx;
    double* vy;
    double* vz;
    double* fx;
    double* fy;
    double* fz;
    double* mass;
    double* inv_mass;
    double* cut;
    uint32_t* tag;
    uint32_t* type;
    int32_t* img;  // 3 planes
    int32_t* origin;
    double* planes[kMaxPlanes];
    int nplanes;
    uint64_t cap;
    // Packed (x, y, z, r) records of the built-in consumer, 4 doubles per
    // atom on a 32-byte boundary (null when unused), r from the plane pkrad
    // of this column set.  The integration pass and forward comm write whole
    // records next to the columns; a packing pass fills them after rebuilds.
    double* pk;
    const double* pkrad;
};

// Where a pass over the atoms also saves the locals' build positions
// (save_build_positions; x == nullptr: not in this pass).
struct BuildPos {
    double* x = nullptr;
    double* y = nullptr;
    double* z = nullptr;
    uint64_t nlocal = 0;
};

// Per-swap constants of the ghost maps (SwapData, comm.rs:114-124).
struct SwapConst {
    double off[kNumSwaps][3];
    double voff[kNumSwaps][3];
};

// Indices of registered f64 planes taking part in an operation.
struct PlaneList {
    int idx[kMaxPlanes];
    int n;
};

// Device-resident counters the host reads back in one copy.
struct DevFlags {
    uint32_t rebuild;        // displacement check tripped
    uint32_t not_identity;   // sort permutation differs from identity
    uint32_t ghost_count[2]; // per-dim lo/hi totals of the last border pass
    uint64_t pairs;          // total pairs of the last count pass
    uint64_t candidates;     // pair candidates tested in the last build
    uint64_t rechecked;      // candidates re-tested in FP64
    uint32_t error;          // device-side guard tripped (index out of range)
    uint32_t fault;          // a bounded device wait ran out (never cleared)
};

}  // namespace soil
