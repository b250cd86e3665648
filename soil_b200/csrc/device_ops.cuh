// device_ops.cuh — per-element device operations shared by the single-system
// kernels and the batched (segmented) kernels, so a box computes exactly the
// same arithmetic whether it runs alone or inside a batch.
#pragma once

#include "kernels.cuh"

namespace soil {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated increment of counts[key] for the valid lanes.
__device__ __forceinline__ void aggregated_count(uint32_t* counts, uint32_t key, bool valid) {
    const uint32_t k = valid ? key : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    const int leader = __ffs(peers) - 1;
    if (valid && (int)(threadIdx.x & 31) == leader) atomicAdd(&counts[key], (uint32_t)__popc(peers));
}

// Displacement test of decide_rebuild (displacement_exceeded, fully periodic
// fast path, neighbor.rs:711-731): nearest image by d - L*round(d/L), FMA sum.
__device__ __forceinline__ bool moved_too_far(double px, double py, double pz, double qx, double qy,
                                              double qz, const double box[3], const double ibox[3],
                                              double thr_sq) {
    double dx = px - qx, dy = py - qy, dz = pz - qz;
    dx -= box[0] * round(dx * ibox[0]);
    dy -= box[1] * round(dy * ibox[1]);
    dz -= box[2] * round(dz * ibox[2]);
    return fma(dx, dx, fma(dy, dy, dz * dz)) > thr_sq;
}

// displacement_exceeded's general path (neighbor.rs:736-756) when some axis
// is not periodic: per-axis single-image correction on periodic axes only.
__device__ __forceinline__ bool moved_too_far_mixed(double px, double py, double pz, double qx,
                                                    double qy, double qz, const double box[3],
                                                    int mask, double thr_sq) {
    double d[3] = {px - qx, py - qy, pz - qz};
    for (int a = 0; a < 3; ++a) {
        if (!(mask & (1 << a))) continue;
        const double h = box[a] * 0.5;
        if (d[a] > h) d[a] -= box[a];
        else if (d[a] < -h) d[a] += box[a];
    }
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > thr_sq;
}

// The displacement check of one local at its new position.
__device__ __forceinline__ bool check_moved_at(const CheckArgs& ck, double x, double y, double z,
                                               double lx, double ly, double lz) {
    if (ck.mask == 7) return moved_too_far(x, y, z, lx, ly, lz, ck.box, ck.ibox, ck.thr_sq);
    return moved_too_far_mixed(x, y, z, lx, ly, lz, ck.box, ck.mask, ck.thr_sq);
}

__device__ __forceinline__ bool check_moved(const CheckArgs& ck, double x, double y, double z,
                                            uint64_t i) {
    return check_moved_at(ck, x, y, z, ck.lbx[i], ck.lby[i], ck.lbz[i]);
}

// wrap_periodic, domain.rs:594-605
__device__ __forceinline__ double wrap1(double p, double low, double sz, int32_t& img) {
    const double high = low + sz;
    if (p < low) {
        img -= 1;
        return p + sz;
    }
    if (p >= high) {
        img += 1;
        return p - sz;
    }
    return p;
}

__device__ __forceinline__ void border_flags(const AtomCols& c, const BorderDim& bd, uint64_t i,
                                             bool& lo, bool& hi) {
    double v;
    if (!bd.triclinic) {
        v = bd.dim == 0 ? c.x[i] : (bd.dim == 1 ? c.y[i] : c.z[i]);
    } else {  // face test in lamda coordinates (comm.rs:305-327)
        double l0, l1, l2;
        x2lamda(bd.geom, c.x[i], c.y[i], c.z[i], l0, l1, l2);
        v = bd.dim == 0 ? l0 : (bd.dim == 1 ? l1 : l2);
    }
    lo = v < bd.thresh_lo;
    hi = v >= bd.thresh_hi;
}

// Face bits of local r for a borders pass: bit 2d = inside the lo slab of
// dim d, bit 2d+1 = inside the hi slab (comm.rs:305-327; lamda coordinates
// when triclinic).
__device__ __forceinline__ uint32_t face_bits(const AtomCols& c, const Geom& geom, int triclinic,
                                              const double* lo, const double* hi, uint64_t r) {
    double v0 = c.x[r], v1 = c.y[r], v2 = c.z[r];
    if (triclinic) {
        double l0, l1, l2;
        x2lamda(geom, v0, v1, v2, l0, l1, l2);
        v0 = l0;
        v1 = l1;
        v2 = l2;
    }
    uint32_t b = 0;
    b |= (v0 < lo[0] ? 1u : 0u) | (v0 >= hi[0] ? 2u : 0u);
    b |= (v1 < lo[1] ? 4u : 0u) | (v1 >= hi[1] ? 8u : 0u);
    b |= (v2 < lo[2] ? 16u : 0u) | (v2 >= hi[2] ? 32u : 0u);
    return b;
}

// Ghost g = image of root r through the swaps of chain category k
// (pack_border + unpack_atom, atom.rs:520-553, applied swap by swap: the
// shifts are added in chain order exactly as the reference's ghost of a
// ghost does); its source (origin) is `parent`.
__device__ __forceinline__ void write_image(const AtomCols& c, const double (*shift)[3],
                                            const double (*vshift)[3], const BorderCats& cats,
                                            int k, uint64_t g, uint64_t r, uint32_t parent,
                                            uint64_t nlocal, uint32_t* root, uint32_t* chain) {
    const uint64_t cap = c.cap;
    double x = c.x[r], y = c.y[r], z = c.z[r];
    double vx = c.vx[r], vy = c.vy[r], vz = c.vz[r];
    uint32_t code = 0;
    for (int t = 0; t < cats.len[k]; ++t) {
        const int s = cats.sw[k][t];
        x = x + shift[s][0];
        y = y + shift[s][1];
        z = z + shift[s][2];
        vx = vx + vshift[s][0];
        vy = vy + vshift[s][1];
        vz = vz + vshift[s][2];
        code |= (uint32_t)s << (3 * t);
    }
    code |= (uint32_t)cats.len[k] << 12;
    // the root's other fields loaded before any store (see perm_gather_atom)
    const double fx = c.fx[r], fy = c.fy[r], fz = c.fz[r];
    const double m = c.mass[r], cu = c.cut[r];
    const uint32_t tg = c.tag[r], ty = c.type[r];
    const int32_t i0 = c.img[r], i1 = c.img[cap + r], i2 = c.img[2 * cap + r];
    c.x[g] = x;
    c.y[g] = y;
    c.z[g] = z;
    c.vx[g] = vx;
    c.vy[g] = vy;
    c.vz[g] = vz;
    c.fx[g] = fx;
    c.fy[g] = fy;
    c.fz[g] = fz;
    c.mass[g] = m;
    c.inv_mass[g] = 1.0 / m;
    c.cut[g] = cu;
    c.tag[g] = tg;
    c.type[g] = ty;
    c.img[g] = i0;
    c.img[cap + g] = i1;
    c.img[2 * cap + g] = i2;
    c.origin[g] = (int32_t)parent;
    for (int q = 0; q < c.nplanes; q += 4) {
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (q + u < c.nplanes) v[u] = c.planes[q + u][r];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (q + u < c.nplanes) c.planes[q + u][g] = v[u];
    }
    root[g - nlocal] = (uint32_t)r;
    chain[g - nlocal] = code;
}

// A sorted record {x, y, z, cutoff} in one 256-bit load through the
// read-only path (the records are written by an earlier launch).
__device__ __forceinline__ double4 ld_rec(const double4* p) {
    double4 v;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
        : "l"(p));
    return v;
}

template <bool UNIFORM, bool FP32>
struct Filter {
    double cut_sq, sf_sq;
    float sf32, eps32, lim_uniform;

    __device__ __forceinline__ explicit Filter(const PairParams& p)
        : cut_sq(p.cut_sq), sf_sq(p.sf_sq), sf32((float)p.sf), eps32(p.eps32), lim_uniform(0.f) {
        if (UNIFORM && FP32) {
            const float cut = (float)sqrt(p.cut_sq) + p.eps32;
            lim_uniform = cut * cut;
        }
    }

    // FP32 prefilter: false only for candidates provably outside the cutoff.
    __device__ __forceinline__ bool pass32(const float4& pif, const float4& q) const {
        const float dx = q.x - pif.x;
        const float dy = q.y - pif.y;
        const float dz = q.z - pif.z;
        const float r2 = dx * dx + dy * dy + dz * dz;
        float lim = lim_uniform;
        if (!UNIFORM) {
            const float cu = (pif.w + q.w) * sf32 + eps32;
            lim = cu * cu;
        }
        return !(r2 > lim);
    }

    // The reference's FP64 test (neighbor.rs:1179-1303): nested FMA distance,
    // uniform cut^2 or (s_i + s_j)^2 * sf^2.
    __device__ __forceinline__ bool test64(const double4& pi, const double4& q) const {
        const double dx = q.x - pi.x;
        const double dy = q.y - pi.y;
        const double dz = q.z - pi.z;
        const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        if (UNIFORM) return r2 < cut_sq;
        const double sum_skin = pi.w + q.w;
        return r2 < sum_skin * sum_skin * sf_sq;
    }

    // The reference pair test for the candidate in sorted slot m; *rechk counts
    // FP64 re-tests in FP32 mode.
    __device__ __forceinline__ bool operator()(const PairParams& p, const double4& pi,
                                               const float4& pif, uint32_t m,
                                               uint32_t* rechk) const {
        if (FP32) {
            if (!pass32(pif, p.spf[m])) return false;
            ++*rechk;
        }
        return test64(pi, ld_rec(p.sp + m));
    }

    // The same test returning the slot's atom when it passes, else kNoAtom.
    // With a uniform cutoff the record's fourth word is free and holds the
    // atom (sorted_view), so the candidate costs one load, not two.
    static constexpr uint32_t kNoAtom = 0xffffffffu;
    __device__ __forceinline__ uint32_t accept(const PairParams& p, const double4& pi,
                                               const float4& pif, uint32_t m,
                                               uint32_t* rechk) const {
        if (!UNIFORM) return (*this)(p, pi, pif, m, rechk) ? p.sorted_atoms[m] : kNoAtom;
        if (FP32) {
            if (!pass32(pif, p.spf[m])) return kNoAtom;
            ++*rechk;
        }
        const double4 q = ld_rec(p.sp + m);
        return test64(pi, q) ? (uint32_t)__double_as_longlong(q.w) : kNoAtom;
    }
};

// Ranges of the row scan held in registers (row_scan_pre): the own cell's
// range and up to kPreRanges - 1 stencil runs.
constexpr int kPreRanges = 8;

// row_scan with every range's slot bounds loaded up front: the own cell's
// range (with newton the tail after i, merged with a first stencil run at
// offset +1, whose cells follow it in slot order) and then each run, held in
// registers and shifted down as ranges are used up, so moving to the next
// range needs no load.  Same candidates in the same order, same counts, as
// row_scan; for stencils of at most kPreRanges - 1 runs.
template <bool UNIFORM, bool FP32, bool FILL>
__device__ uint32_t row_scan_pre(const PairParams& p, const Filter<UNIFORM, FP32>& test,
                                 uint64_t i, uint32_t* out, uint32_t cap, uint32_t* rechk,
                                 uint32_t* cand, DevFlags* flags, uint32_t* in_count) {
    const uint32_t my_cell = p.atom_cell[i];
    const uint32_t mi = p.atom_sorted_idx[i];
    const double4 pi = ld_rec(p.sp + mi);
    const float4 pif = FP32 ? p.spf[mi] : make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t rm[kPreRanges], re[kPreRanges];
    int first = 0;  // stencil runs merged into the own range
    rm[0] = 0;
    re[0] = 0;
    if (p.has_self) {
        uint64_t ce = (uint64_t)my_cell + 1;
        if (p.newton && p.nstencil > 0 && p.stencil[0] == 1 &&
            ce + (uint64_t)p.stencil[1] <= p.ncells) {
            ce += (uint64_t)p.stencil[1];
            first = 1;
        }
        rm[0] = p.newton ? mi + 1 : p.bin_start[my_cell];
        re[0] = p.bin_start[ce];
    }
    uint32_t total = re[0] - rm[0];
#pragma unroll
    for (int k = 1; k < kPreRanges; ++k) {
        rm[k] = 0;
        re[k] = 0;
        const int s = first + k - 1;
        if (s < p.nstencil) {
            const int64_t c0 = (int64_t)my_cell + p.stencil[2 * s];
            const int64_t c1 = c0 + p.stencil[2 * s + 1];
            if (c0 < 0 || c1 > (int64_t)p.ncells) {  // the grid's ghost layers make this unreachable
                if (flags) atomicOr(&flags->error, 1u);
            } else {
                rm[k] = p.bin_start[c0];
                re[k] = p.bin_start[c1];
                total += re[k] - rm[k];
            }
        }
    }
    const bool skip_i = p.has_self && !p.newton;  // i is in its own range
    *cand += total - (skip_i ? 1u : 0u);
    int left = 1 + (p.nstencil - first);  // ranges not yet finished, the current one included
    bool own = true;
    uint32_t cnt = 0;
    uint32_t m = rm[0], e = re[0];
    for (;;) {
        while (m >= e) {  // the next range, shifted in from the registers
            if (--left <= 0) return cnt;
#pragma unroll
            for (int k = 0; k + 1 < kPreRanges; ++k) {
                rm[k] = rm[k + 1];
                re[k] = re[k + 1];
            }
            m = rm[0];
            e = re[0];
            own = false;
        }
        if (own && skip_i && m == mi) {
            ++m;
            continue;
        }
        // the candidate's atom, loaded with its record rather than after the
        // test accepts it (a dependent round trip per accepted entry)
        uint32_t a;
        bool ok;
        if (UNIFORM) {  // the atom comes with the record
            a = test.accept(p, pi, pif, m, rechk);
            ok = a != test.kNoAtom;
        } else {
            a = p.sorted_atoms[m];
            ok = test(p, pi, pif, m, rechk);
        }
        if (ok) {
            if (in_count) atomicAdd(&in_count[a], 1u);
            if (FILL && cnt < cap) out[cnt] = a;
            ++cnt;
        }
        ++m;
    }
}

// Row of local atom i, sequentially in reference order: the own cell's
// candidates (the tail after i's slot with newton, else the whole cell
// without i), then every stencil cell in stencil order, each in sorted order.
// The stencil comes as runs of consecutive cells (p.stencil holds (offset,
// cells) pairs, p.nstencil runs; stencil_runs on the host): the offsets
// ascend, so a run's cells are one contiguous range of sorted slots and the
// order is the cell-by-cell order.  The candidate ranges run as ONE loop (the
// lane moves to its next non-empty range when one ends), so a warp pays for
// the longest candidate sequence of its lanes rather than the per-cell
// maximum summed over the stencil.  FILL writes the accepted indices to out[]
// (at most cap); in_count (optional) counts every accepted index.  Returns
// the row length.
template <bool UNIFORM, bool FP32, bool FILL>
__device__ uint32_t row_scan(const PairParams& p, const Filter<UNIFORM, FP32>& test, uint64_t i,
                             uint32_t* out, uint32_t cap, uint32_t* rechk, uint32_t* cand,
                             DevFlags* flags, uint32_t* in_count = nullptr) {
    if (p.pre_ranges && p.nstencil < kPreRanges)
        return row_scan_pre<UNIFORM, FP32, FILL>(p, test, i, out, cap, rechk, cand, flags,
                                                 in_count);
    const uint32_t my_cell = p.atom_cell[i];
    const uint32_t mi = p.atom_sorted_idx[i];
    const double4 pi = ld_rec(p.sp + mi);
    const float4 pif = FP32 ? p.spf[mi] : make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t cnt = 0;
    int s = -1;  // -1: the own cell; s >= 0: stencil cell s
    uint32_t m = 0, e = 0;
    if (p.has_self) {
        e = p.bin_start[my_cell + 1];
        m = p.newton ? mi + 1 : p.bin_start[my_cell];
    }
    for (;;) {
        while (m >= e) {  // open the next non-empty run of stencil cells
            if (++s >= p.nstencil) return cnt;
            const int64_t c0 = (int64_t)my_cell + p.stencil[2 * s];
            const int64_t c1 = c0 + p.stencil[2 * s + 1];  // one past its last cell
            if (c0 < 0 || c1 > (int64_t)p.ncells) {  // the grid's ghost layers make this unreachable
                if (flags) atomicOr(&flags->error, 1u);
                continue;
            }
            m = p.bin_start[c0];
            e = p.bin_start[c1];
            *cand += e - m;
        }
        if (s < 0) {  // own cell: i itself is not a candidate
            if (!p.newton && m == mi) {
                ++m;
                continue;
            }
            ++*cand;
        }
        const uint32_t a = test.accept(p, pi, pif, m, rechk);
        if (a != test.kNoAtom) {
            if (in_count) atomicAdd(&in_count[a], 1u);  // pass 1 of a build with the transposed lists
            if (FILL && cnt < cap) out[cnt] = a;
            ++cnt;
        }
        ++m;
    }
}

// ---- per-atom bodies of the kernels ----------------------------------------

// Atom i's packed record (x, y, z, its radius) in one 256-bit store: whole
// 32-byte sectors, so the write needs no read of the old record.  The radius
// is atom i's value of the plane c.pkrad (a forward comm copies a ghost's
// forward planes before it writes the record).
__device__ __forceinline__ void put_pk(double* pk, uint64_t i, double x, double y, double z,
                                       double r) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};"
                 :
                 : "l"(pk + 4 * i), "d"(x), "d"(y), "d"(z), "d"(r)
                 : "memory");
}

// Atom i's packed record (32-byte aligned) in one 256-bit load.  A plain
// (coherent) load: the resident steps write the records between their grid
// barriers, so the non-coherent path is not an option; the memory clobber
// keeps the load in program order with the kernel's other accesses.
__device__ __forceinline__ double4 ld_pk(const double* pk, uint64_t i) {
    double4 v;
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
                 : "l"(pk + 4 * i)
                 : "memory");
    return v;
}

// initial_integration (soil_verlet/src/lib.rs:131-162) on registers: v += h*F
// (twice when fuse_final: the previous step's final_integration with the same
// forces first), then x += v*dt; h = dt/2 * inv_mass.
__device__ __forceinline__ void initial_regs(double h, double dt, bool fuse_final, double fx,
                                             double fy, double fz, double& vx, double& vy,
                                             double& vz, double& x, double& y, double& z) {
    if (fuse_final) {
        vx = vx + h * fx;
        vy = vy + h * fy;
        vz = vz + h * fz;
    }
    vx = vx + h * fx;
    vy = vy + h * fy;
    vz = vz + h * fz;
    x = x + vx * dt;
    y = y + vy * dt;
    z = z + vz * dt;
}

// initial_integration (soil_verlet/src/lib.rs:131-162) of atom i, optionally
// preceded by final_integration of the previous step with the same forces;
// returns the new position.
__device__ __forceinline__ void initial_atom(const AtomCols& c, uint64_t i, double dt,
                                             bool fuse_final, bool zero_force, double& x,
                                             double& y, double& z, double& v0, double& v1,
                                             double& v2) {
    // every load first: a load after this atom's stores could not be moved
    // above them (the compiler cannot tell the columns apart) and would cost
    // another memory round trip
    const double h = 0.5 * dt * c.inv_mass[i];
    const double fx = c.fx[i], fy = c.fy[i], fz = c.fz[i];
    v0 = c.vx[i];
    v1 = c.vy[i];
    v2 = c.vz[i];
    x = c.x[i];
    y = c.y[i];
    z = c.z[i];
    initial_regs(h, dt, fuse_final, fx, fy, fz, v0, v1, v2, x, y, z);
    c.vx[i] = v0;
    c.vy[i] = v1;
    c.vz[i] = v2;
    c.x[i] = x;
    c.y[i] = y;
    c.z[i] = z;
    if (c.pk) put_pk(c.pk, i, x, y, z, c.pkrad[i]);
    if (zero_force) {  // zero_all_forces, atom.rs:631-635 (locals part)
        c.fx[i] = 0.0;
        c.fy[i] = 0.0;
        c.fz[i] = 0.0;
    }
}

__device__ __forceinline__ void initial_atom(const AtomCols& c, uint64_t i, double dt,
                                             bool fuse_final, bool zero_force, double& x,
                                             double& y, double& z) {
    double v0, v1, v2;
    initial_atom(c, i, dt, fuse_final, zero_force, x, y, z, v0, v1, v2);
}

// final_integration, soil_verlet/src/lib.rs:175-194: v += h*F
__device__ __forceinline__ void final_atom(const AtomCols& c, uint64_t i, double dt) {
    const double h = 0.5 * dt * c.inv_mass[i];
    c.vx[i] = c.vx[i] + h * c.fx[i];
    c.vy[i] = c.vy[i] + h * c.fy[i];
    c.vz[i] = c.vz[i] + h * c.fz[i];
}

// pbc fully periodic fast path (domain.rs:626-636) / pbc_triclinic
// (domain.rs:674-729) of a position held in registers: wrapped in place, the
// image counts updated, and remap(s) called with the y crossing s (+1 / -1)
// for the Lees–Edwards velocity remap v -= s * bvel.
template <class Remap>
__device__ __forceinline__ void pbc_core(const Geom& g, double& x, double& y, double& z,
                                         int32_t& i0, int32_t& i1, int32_t& i2, Remap remap) {
    if (!g.triclinic) {
        x = wrap1(x, g.lo[0], g.size[0], i0);
        y = wrap1(y, g.lo[1], g.size[1], i1);
        z = wrap1(z, g.lo[2], g.size[2], i2);
        return;
    }
    double l0, l1, l2;
    x2lamda(g, x, y, z, l0, l1, l2);
    int32_t d0 = 0, d1 = 0, d2 = 0;
    if (l0 < 0.0) { l0 += 1.0; d0 = -1; } else if (l0 >= 1.0) { l0 -= 1.0; d0 = 1; }
    if (l1 < 0.0) { l1 += 1.0; d1 = -1; } else if (l1 >= 1.0) { l1 -= 1.0; d1 = 1; }
    if (l2 < 0.0) { l2 += 1.0; d2 = -1; } else if (l2 >= 1.0) { l2 -= 1.0; d2 = 1; }
    lamda2x(g, l0, l1, l2, x, y, z);
    i0 += d0;
    i1 += d1;
    i2 += d2;
    if (d1 != 0) remap((double)d1);
}

// pbc of local i in memory; the new position also into px, py, pz
__device__ __forceinline__ void pbc_atom(const AtomCols& c, uint64_t i, const Geom& g, double bv0,
                                         double bv1, double bv2, double& px, double& py,
                                         double& pz) {
    const uint64_t cap = c.cap;
    int32_t i0 = c.img[i], i1 = c.img[cap + i], i2 = c.img[2 * cap + i];
    px = c.x[i];
    py = c.y[i];
    pz = c.z[i];
    pbc_core(g, px, py, pz, i0, i1, i2, [&](double s) {
        c.vx[i] = c.vx[i] - s * bv0;
        c.vy[i] = c.vy[i] - s * bv1;
        c.vz[i] = c.vz[i] - s * bv2;
    });
    c.x[i] = px;
    c.y[i] = py;
    c.z[i] = pz;
    c.img[i] = i0;
    c.img[cap + i] = i1;
    c.img[2 * cap + i] = i2;
}

__device__ __forceinline__ void pbc_atom(const AtomCols& c, uint64_t i, const Geom& g, double bv0,
                                         double bv1, double bv2) {
    double px, py, pz;
    pbc_atom(c, i, g, bv0, bv1, bv2, px, py, pz);
}

// forward_comm of ghost gi (index nlocal + gi): its root local atom plus the
// offsets of its swap chain, added in chain order (comm.rs:400-432).
__device__ __forceinline__ void forward_ghost(const AtomCols& c, uint64_t nlocal, uint64_t gi,
                                              const uint32_t* root, const uint32_t* chain,
                                              const SwapConst& sc, const PlaneList& fwd,
                                              bool zero_force) {
    const uint64_t g = nlocal + gi;
    const uint32_t r = root[gi];
    const uint32_t code = chain[gi];
    const uint32_t len = code >> 12;
    double px = c.x[r], py = c.y[r], pz = c.z[r];
    double vx = c.vx[r], vy = c.vy[r], vz = c.vz[r];
    for (uint32_t k = 0; k < len; ++k) {
        const int s = (code >> (3 * k)) & 7;
        px = px + sc.off[s][0];
        py = py + sc.off[s][1];
        pz = pz + sc.off[s][2];
        vx = vx + sc.voff[s][0];
        vy = vy + sc.voff[s][1];
        vz = vz + sc.voff[s][2];
    }
    c.x[g] = px;
    c.y[g] = py;
    c.z[g] = pz;
    c.vx[g] = vx;
    c.vy[g] = vy;
    c.vz[g] = vz;
    for (int q = 0; q < fwd.n; ++q) c.planes[fwd.idx[q]][g] = c.planes[fwd.idx[q]][r];
    if (c.pk) put_pk(c.pk, g, px, py, pz, c.pkrad[g]);  // after the planes: g's own radius
    if (zero_force) {
        c.fx[g] = 0.0;
        c.fy[g] = 0.0;
        c.fz[g] = 0.0;
    }
}

// forward_comm of every image of local r, from r's new position and velocity
// (held by the caller): the same additions as forward_ghost, in chain order,
// for the ghosts of r's fold program.
__device__ __forceinline__ void forward_images(const AtomCols& c, uint64_t nlocal, uint64_t r,
                                               double px0, double py0, double pz0, double vx0,
                                               double vy0, double vz0, const uint32_t* fold_start,
                                               const uint32_t* fold_list, const uint32_t* chain,
                                               const SwapConst& sc, const PlaneList& fwd,
                                               bool zero_force) {
    const uint32_t f1 = fold_start[r + 1];
    for (uint32_t f = fold_start[r]; f < f1; ++f) {
        const uint32_t gi = fold_list[f];
        const uint64_t g = nlocal + gi;
        const uint32_t code = chain[gi];
        const uint32_t len = code >> 12;
        double px = px0, py = py0, pz = pz0, vx = vx0, vy = vy0, vz = vz0;
        for (uint32_t k = 0; k < len; ++k) {
            const int s = (code >> (3 * k)) & 7;
            px = px + sc.off[s][0];
            py = py + sc.off[s][1];
            pz = pz + sc.off[s][2];
            vx = vx + sc.voff[s][0];
            vy = vy + sc.voff[s][1];
            vz = vz + sc.voff[s][2];
        }
        c.x[g] = px;
        c.y[g] = py;
        c.z[g] = pz;
        c.vx[g] = vx;
        c.vy[g] = vy;
        c.vz[g] = vz;
        for (int q = 0; q < fwd.n; ++q) c.planes[fwd.idx[q]][g] = c.planes[fwd.idx[q]][r];
        if (c.pk) put_pk(c.pk, g, px, py, pz, c.pkrad[g]);  // after the planes: g's own radius
        if (zero_force) {
            c.fx[g] = 0.0;
            c.fy[g] = 0.0;
            c.fz[g] = 0.0;
        }
    }
}

// Force on atom a from the built-in consumer, in the reference's summation
// order: -f(i,a) for every earlier row i listing a (ascending i), then
// +f(a,j) over a's own row, then -f(i,a) for later rows (ghost atoms and, with
// newton off, non-receiving atoms skip parts).  The three parts run as ONE
// loop over the flattened sequence (in-list entries below a, the row, the
// rest of the in-list), so a warp pays the longest sequence of its lanes, not
// the sum of three per-part maxima.  Each entry evaluates f(i, j) with i the
// row atom, with the same operations in the same order, so the sums are
// bit-identical to the sequential reference.  f(i, j) is the tutorial's
// soft_repulsion_force (docs/src/tutorial/write-your-own-physics.md:56-110):
// d = x_j - x_i, overlap = (r_i + r_j) - |d|, f_i = -K * overlap * d / |d|.
__device__ __forceinline__ void harmonic_atom(const AtomCols& c, uint64_t a, uint64_t nlocal,
                                              const double* rad, double K, int newton,
                                              const uint32_t* offsets, const uint32_t* indices,
                                              const uint32_t* in_start, const uint32_t* in_list) {
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    const bool local = a < nlocal;
    // reference applies -f to j only when newton || j < nlocal
    const bool receives = newton || local;
    const uint32_t qs = in_start[a];
    const uint32_t nin = receives ? in_start[a + 1] - qs : 0u;
    const uint32_t rs = local ? offsets[a] : 0u;
    const uint32_t nrow = local ? offsets[a + 1] - rs : 0u;
    uint32_t npre = 0;  // in-list rows below a (the list is ascending, never a itself)
    while (npre < nin && in_list[qs + npre] < (uint32_t)a) ++npre;
    const double xa = c.x[a], ya = c.y[a], za = c.z[a], ra = rad[a];
    const uint32_t total = nin + nrow;
    for (uint32_t k = 0; k < total; ++k) {
        const bool own = k >= npre && k < npre + nrow;
        const uint32_t o = own ? indices[rs + (k - npre)] : in_list[qs + (k < npre ? k : k - nrow)];
        const double xo = c.x[o], yo = c.y[o], zo = c.z[o], ro = rad[o];
        // f(i, j): own row i = a, j = o; in-list i = o, j = a
        const double ri = own ? ra : ro, rj = own ? ro : ra;
        const double xi = own ? xa : xo, xj = own ? xo : xa;
        const double yi = own ? ya : yo, yj = own ? yo : ya;
        const double zi = own ? za : zo, zj = own ? zo : za;
        const double sum_r = ri + rj;
        const double dx = xj - xi;
        const double dy = yj - yi;
        const double dz = zj - zi;
        const double dist_sq = dx * dx + dy * dy + dz * dz;
        if (dist_sq >= sum_r * sum_r || dist_sq == 0.0) continue;
        const double dist = sqrt(dist_sq);
        const double overlap = sum_r - dist;
        const double inv_dist = 1.0 / dist;
        const double fmag = K * overlap;
        const double fx = -fmag * dx * inv_dist;
        const double fy = -fmag * dy * inv_dist;
        const double fz = -fmag * dz * inv_dist;
        if (own) {
            Fx = Fx + fx;
            Fy = Fy + fy;
            Fz = Fz + fz;
        } else {
            Fx = Fx - fx;
            Fy = Fy - fy;
            Fz = Fz - fz;
        }
    }
    c.fx[a] = Fx;
    c.fy[a] = Fy;
    c.fz[a] = Fz;
}

// reverse_send_force for the image tree of local atom t, in fold order.
__device__ __forceinline__ void fold_root(const AtomCols& c, uint64_t nlocal, uint64_t t,
                                          const uint32_t* start, const uint32_t* list,
                                          const PlaneList& rev) {
    const uint32_t b = start[t], e = start[t + 1];
    for (uint32_t q = b; q < e; ++q) {
        const uint64_t g = nlocal + list[q];
        const uint32_t o = (uint32_t)c.origin[g];
        c.fx[o] = c.fx[o] + c.fx[g];
        c.fy[o] = c.fy[o] + c.fy[g];
        c.fz[o] = c.fz[o] + c.fz[g];
        for (int k = 0; k < rev.n; ++k)
            c.planes[rev.idx[k]][o] = c.planes[rev.idx[k]][o] + c.planes[rev.idx[k]][g];
    }
}

// one sorted slot of the neighbor build's bin order (neighbor.rs:1101-1125)
__device__ __forceinline__ void sorted_view(const AtomCols& c, uint64_t m, const uint32_t* sorted,
                                            uint32_t* asi, double4* sp, float4* spf, double o0,
                                            double o1, double o2, const BuildPos& bp = BuildPos{},
                                            bool atom_in_w = false) {
    const uint32_t a = sorted[m];
    asi[a] = (uint32_t)m;
    const double x = c.x[a], y = c.y[a], z = c.z[a], cut = c.cut[a];
    // with a uniform cutoff the pair test reads no radius: the fourth word
    // carries the slot's atom instead (its bits; Filter::accept)
    sp[m] = make_double4(x, y, z, atom_in_w ? __longlong_as_double((long long)a) : cut);
    if (spf) spf[m] = make_float4((float)(x - o0), (float)(y - o1), (float)(z - o2), (float)cut);
    if (bp.x && a < bp.nlocal) {  // save_build_positions of the locals
        bp.x[a] = x;
        bp.y[a] = y;
        bp.z[a] = z;
    }
}

// Restore ascending order of one segment (the stable counting sort's last
// step) and return how many of its items are below `pivot`: segments of up
// to 8 items (nearly all: bins and transposed lists hold a few atoms) are
// loaded at once and sorted in registers by an odd-even transposition
// network, the count taken from the registers; longer ones are sorted by
// insertion in place.  The items of a segment are distinct, so the order is
// unique.
__device__ __forceinline__ uint32_t sort_segment(uint32_t* items, uint32_t b, uint32_t e,
                                                 uint32_t pivot) {
    const uint32_t n = e - b;
    if (n == 0) return 0;
    if (n <= 8) {
        uint32_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = (uint32_t)k < n ? items[b + k] : 0xffffffffu;
        if (n >= 2) {
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int k = r & 1; k + 1 < 8; k += 2) {
                    const uint32_t lo = min(v[k], v[k + 1]), hi = max(v[k], v[k + 1]);
                    v[k] = lo;
                    v[k + 1] = hi;
                }
        }
        uint32_t below = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if ((uint32_t)k < n) {
                if (n >= 2) items[b + k] = v[k];
                below += v[k] < pivot;
            }
        return below;
    }
    for (uint32_t k = b + 1; k < e; ++k) {
        const uint32_t v = items[k];
        uint32_t j = k;
        while (j > b && items[j - 1] > v) {
            items[j] = items[j - 1];
            --j;
        }
        items[j] = v;
    }
    uint32_t k = b;
    while (k < e && items[k] < pivot) ++k;
    return k - b;
}

// restore ascending order of one segment
__device__ __forceinline__ void insertion_sort(uint32_t* items, uint32_t b, uint32_t e) {
    if (e - b >= 2) sort_segment(items, b, e, 0u);
}

// one atom of the spatial sort's permutation gather (atom.rs:479-490)
// (forces: false when this step's consumer overwrites every force before
// anything reads one, so the old values need not move)
__device__ __forceinline__ void perm_gather_atom(const AtomCols& s, const AtomCols& d, uint64_t k,
                                                 uint32_t p, bool forces = true) {
    const uint64_t cap = s.cap, dcap = d.cap;
    // Every load before any store: the compiler cannot prove the two column
    // sets apart, so interleaved loads and stores would make each thread wait
    // out one memory round trip per column.
    const double x = s.x[p], y = s.y[p], z = s.z[p];
    const double vx = s.vx[p], vy = s.vy[p], vz = s.vz[p];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    if (forces) {
        fx = s.fx[p];
        fy = s.fy[p];
        fz = s.fz[p];
    }
    const double m = s.mass[p], im = s.inv_mass[p], cu = s.cut[p];
    const uint32_t tg = s.tag[p], ty = s.type[p];
    const int32_t i0 = s.img[p], i1 = s.img[cap + p], i2 = s.img[2 * cap + p];
    const int32_t org = s.origin[p];
    d.x[k] = x;
    d.y[k] = y;
    d.z[k] = z;
    d.vx[k] = vx;
    d.vy[k] = vy;
    d.vz[k] = vz;
    if (forces) {
        d.fx[k] = fx;
        d.fy[k] = fy;
        d.fz[k] = fz;
    }
    d.mass[k] = m;
    d.inv_mass[k] = im;
    d.cut[k] = cu;
    d.tag[k] = tg;
    d.type[k] = ty;
    d.img[k] = i0;
    d.img[dcap + k] = i1;
    d.img[2 * dcap + k] = i2;
    d.origin[k] = org;
    for (int q = 0; q < s.nplanes; q += 4) {  // four planes' loads, then their stores
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (q + u < s.nplanes) v[u] = s.planes[q + u][p];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (q + u < s.nplanes) d.planes[q + u][k] = v[u];
    }
}

}  // namespace soil
