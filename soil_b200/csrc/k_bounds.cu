// k_bounds.cu — non-periodic and shrink-wrapped boundaries (domain.rs:509-663):
// the wrap-or-remove pass of pbc, ordered selection of flagged atoms (atoms to
// remove, or atoms at a face that has no neighbor to send to), and the extent
// of the locals along shrink-wrapped axes.
#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

// pbc slow path (domain.rs:641-662) for one atom: periodic axes wrap, an axis
// without periodicity flags the atom for removal when it lies outside [lo, hi).
__global__ void __launch_bounds__(kBlock) k_pbc_bounded(uint64_t n, AtomCols c, BoundsArgs b,
                                                        uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t gone = 0;
        for (int d = 0; d < 3 && !gone; ++d) {
            double* x = d == 0 ? c.x : d == 1 ? c.y : c.z;
            int32_t* img = c.img + (uint64_t)d * c.cap;
            if (b.periodic & (1 << d)) {
                int32_t im = img[i];
                x[i] = wrap1(x[i], b.lo[d], b.size[d], im);
                img[i] = im;
            } else if (x[i] < b.lo[d] || x[i] >= b.hi[d]) {
                gone = 1;
            }
        }
        out[i] = gone;
    }
}

// pbc_triclinic (domain.rs:673-729) with fixed axes: periodic axes wrap in
// lamda space (with the Lees–Edwards velocity remap on a y crossing), an atom
// outside [0, 1) of a fixed axis is flagged; kept atoms are rewritten from
// lamda as in the all-periodic path.
__global__ void __launch_bounds__(kBlock) k_pbc_bounded_tri(uint64_t n, AtomCols c, Geom g,
                                                            int periodic, double bv0, double bv1,
                                                            double bv2, uint32_t* out) {
    const uint64_t cap = c.cap;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double l[3];
        x2lamda(g, c.x[i], c.y[i], c.z[i], l[0], l[1], l[2]);
        int32_t dl[3] = {0, 0, 0};
        uint32_t gone = 0;
        for (int d = 0; d < 3 && !gone; ++d) {
            if (periodic & (1 << d)) {
                if (l[d] < 0.0) { l[d] += 1.0; dl[d] = -1; }
                else if (l[d] >= 1.0) { l[d] -= 1.0; dl[d] = 1; }
            } else if (l[d] < 0.0 || l[d] >= 1.0) {
                gone = 1;
            }
        }
        out[i] = gone;
        if (gone) continue;
        double rx, ry, rz;
        lamda2x(g, l[0], l[1], l[2], rx, ry, rz);
        c.x[i] = rx;
        c.y[i] = ry;
        c.z[i] = rz;
        for (int d = 0; d < 3; ++d) c.img[d * cap + i] += dl[d];
        if (dl[1] != 0) {
            const double s = (double)dl[1];
            c.vx[i] = c.vx[i] - s * bv0;
            c.vy[i] = c.vy[i] - s * bv1;
            c.vz[i] = c.vz[i] - s * bv2;
        }
    }
}

void launch_pbc_bounded(cudaStream_t st, uint64_t n, const AtomCols& c, const BoundsArgs& b,
                        uint32_t* gone) {
    if (n == 0) return;
    note_launch();
    if (b.geom.triclinic)
        k_pbc_bounded_tri<<<grid_for(n), kBlock, 0, st>>>(n, c, b.geom, b.periodic, b.bvel[0],
                                                          b.bvel[1], b.bvel[2], gone);
    else
        k_pbc_bounded<<<grid_for(n), kBlock, 0, st>>>(n, c, b, gone);
}

// pack_border_atoms' face test (comm.rs:305-358): flag[i] for atoms [0, n) at
// the low (side 0: v < thresh) or high (v >= thresh) face of axis dim, with v
// the coordinate, or its lamda value when the box is triclinic.
__global__ void __launch_bounds__(kBlock) k_face_flag(uint64_t n, AtomCols c, Geom g, int dim,
                                                      double thresh, int side, uint32_t* flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double v;
        if (g.triclinic) {
            double l0, l1, l2;
            x2lamda(g, c.x[i], c.y[i], c.z[i], l0, l1, l2);
            v = dim == 0 ? l0 : dim == 1 ? l1 : l2;
        } else {
            v = dim == 0 ? c.x[i] : dim == 1 ? c.y[i] : c.z[i];
        }
        flag[i] = side == 0 ? (v < thresh) : (v >= thresh);
    }
}

void launch_face_flag(cudaStream_t st, uint64_t n, const AtomCols& c, const Geom& g, int dim,
                      double thresh, int side, uint32_t* flag) {
    if (n == 0) return;
    note_launch();
    k_face_flag<<<grid_for(n), kBlock, 0, st>>>(n, c, g, dim, thresh, side, flag);
}

__global__ void __launch_bounds__(kBlock) k_scatter_selected(uint64_t n, const uint32_t* flag,
                                                             const uint32_t* pos, uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        if (flag[i]) out[pos[i]] = (uint32_t)i;
}

void launch_select(cudaStream_t st, uint64_t n, const uint32_t* flag, uint32_t* pos,
                   uint32_t* temp, uint32_t* out) {
    exclusive_scan_u32(st, flag, pos, n, temp);
    if (n == 0) return;
    note_launch();
    k_scatter_selected<<<grid_for(n), kBlock, 0, st>>>(n, flag, pos, out);
}

// Order-preserving u64 key of a double (min/max of keys = min/max of values).
__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// ext[d] = min key, ext[3 + d] = max key of x_d over [0, n) for axes in mask.
__global__ void __launch_bounds__(kBlock) k_extent(uint64_t n, AtomCols c, int mask,
                                                   unsigned long long* ext) {
    unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (int d = 0; d < 3; ++d) {
            if (!(mask & (1 << d))) continue;
            const unsigned long long k = order_key(d == 0 ? c.x[i] : d == 1 ? c.y[i] : c.z[i]);
            mn[d] = k < mn[d] ? k : mn[d];
            mx[d] = k > mx[d] ? k : mx[d];
        }
    for (int d = 0; d < 3; ++d) {
        if (!(mask & (1 << d))) continue;
        unsigned long long a = mn[d], z = mx[d];
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long a2 = __shfl_xor_sync(0xffffffffu, a, o);
            const unsigned long long z2 = __shfl_xor_sync(0xffffffffu, z, o);
            a = a2 < a ? a2 : a;
            z = z2 > z ? z2 : z;
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&ext[d], a);
            atomicMax(&ext[3 + d], z);
        }
    }
}

void launch_extent(cudaStream_t st, uint64_t n, const AtomCols& c, int mask,
                   unsigned long long* ext) {
    if (n == 0) return;
    note_launch();
    k_extent<<<grid_for(n), kBlock, 0, st>>>(n, c, mask, ext);
}

}  // namespace soil
