// force_ops.cuh — the grouped built-in consumer's warp tile (device code
// shared by the one-launch consumer k_force_seq and the device-resident
// multi-step kernel k_steps).  How the tile reproduces the reference's force
// sums is described at the top of k_force.cu.
#pragma once

#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

// ---- the grouped partner sequences (rebuilt with the lists) ----------------

// Entries of atom a in the reference sum: its in-list (when it receives:
// newton, or a local) and its own row (locals).
__device__ __forceinline__ uint32_t seq_len(uint64_t a, uint64_t nlocal, int newton,
                                            const uint32_t* offsets, const uint32_t* in_start) {
    const bool local = a < nlocal;
    const uint32_t nin = (newton || local) ? in_start[a + 1] - in_start[a] : 0u;
    const uint32_t nrow = local ? offsets[a + 1] - offsets[a] : 0u;
    return nin + nrow;
}

// cnt[a] = entries of atom a (every atom); grp[t] = entries of root t's group
// (t and its images), t < nlocal.
__device__ __forceinline__ void seq_count_atom(const SeqArgs& q, uint64_t a, uint32_t* cnt,
                                               uint32_t* grp) {
    const uint32_t n = seq_len(a, q.nlocal, q.newton, q.offsets, q.in_start);
    cnt[a] = n;
    if (a < q.nlocal) {
        uint32_t g = n;
        for (uint32_t f = q.fold_start[a]; f < q.fold_start[a + 1]; ++f)
            g += seq_len(q.nlocal + q.fold_list[f], q.nlocal, q.newton, q.offsets, q.in_start);
        grp[a] = g;
    }
}

// The entries of atom a from position k on: in-list rows below a
// (ascending), a's own row in CSR order, then the in-list rows above a.
__device__ __forceinline__ uint32_t seq_put(const SeqArgs& q, uint64_t a, uint32_t k,
                                            uint8_t meta, uint32_t* seq, uint8_t* owner) {
    const bool local = a < q.nlocal;
    const uint32_t qs = q.in_start[a];
    const uint32_t nin = (q.newton || local) ? q.in_start[a + 1] - qs : 0u;
    const uint32_t rs = local ? q.offsets[a] : 0u;
    const uint32_t nrow = local ? q.offsets[a + 1] - rs : 0u;
    uint32_t i = 0;
    for (; i < nin && q.in_list[qs + i] < (uint32_t)a; ++i, ++k) {
        seq[k] = q.in_list[qs + i];
        owner[k] = meta;
    }
    for (uint32_t r = 0; r < nrow; ++r, ++k) {
        seq[k] = q.indices[rs + r];
        owner[k] = meta;
    }
    for (; i < nin; ++i, ++k) {
        seq[k] = q.in_list[qs + i];
        owner[k] = meta;
    }
    return k;
}

// Group of root t at grp_start[t]: t's entries, then each image's in fold
// order.  owner[k] = (t & 31) | item << 5: item 0 = the root, item j = its
// j-th image (at most 7 images per root, which the host checks).
__device__ __forceinline__ void seq_fill_root(const SeqArgs& q, uint64_t t,
                                              const uint32_t* grp_start, uint32_t* seq,
                                              uint8_t* owner) {
    const uint8_t lane = (uint8_t)(t & 31);
    uint32_t k = seq_put(q, t, grp_start[t], lane, seq, owner);
    const uint32_t f0 = q.fold_start[t], f1 = q.fold_start[t + 1];
    for (uint32_t f = f0; f < f1; ++f)
        k = seq_put(q, q.nlocal + q.fold_list[f], k, (uint8_t)(lane | ((f - f0 + 1) << 5)), seq,
                    owner);
}

// ---- the warp tile ------------------------------------------------------------

constexpr int kForceWarps = kBlock / 32;

template <int U>
struct ForceSmem {
    double fx[kForceWarps][32 * U];
    double fy[kForceWarps][32 * U];
    double fz[kForceWarps][32 * U];
    uint32_t hit[kForceWarps][U];  // contact ballots of the chunk's rows
};

// f(i, j) of the tutorial consumer with i = a (the owner) and j = o
// (docs/src/tutorial/write-your-own-physics.md:56-110).
__device__ __forceinline__ bool pair_force(double xa, double ya, double za, double ra, double xo,
                                           double yo, double zo, double ro, double K, double& fx,
                                           double& fy, double& fz) {
    const double sum_r = ra + ro;
    const double dx = xo - xa;
    const double dy = yo - ya;
    const double dz = zo - za;
    const double dist_sq = dx * dx + dy * dy + dz * dz;
    if (dist_sq >= sum_r * sum_r || dist_sq == 0.0) return false;
    const double dist = sqrt(dist_sq);
    const double overlap = sum_r - dist;
    const double inv_dist = 1.0 / dist;
    const double fmag = K * overlap;
    fx = -fmag * dx * inv_dist;
    fy = -fmag * dy * inv_dist;
    fz = -fmag * dz * inv_dist;
    return true;
}

// Partner records for the one-thread-per-root walks: the packed copy (one
// 256-bit load) or the x, y, z and radius columns (four loads).
struct PkLd {
    const double* pk;
    __device__ __forceinline__ double4 operator()(uint64_t o) const { return ld_pk(pk, o); }
};
struct ColLd {
    const double* x;
    const double* y;
    const double* z;
    const double* r;
    __device__ __forceinline__ double4 operator()(uint64_t o) const {
        return make_double4(x[o], y[o], z[o], r[o]);
    }
};

// F += f(a, o) over the partners o = idx(0), ..., idx(n - 1) in that order.
// Partner k + 1's record is loaded before partner k's force is evaluated, so
// two gathers are in flight per thread (deeper lookahead measured slower: it
// costs registers and occupancy).
template <class Ld, class Idx>
__device__ __forceinline__ void sum_partners(const Ld& ld, const double4& pa, double K, uint32_t n,
                                             const Idx& idx, double& Fx, double& Fy, double& Fz) {
    if (n == 0) return;
    double4 cur = ld(idx(0));
    for (uint32_t k = 0; k < n; ++k) {
        double4 nxt = cur;
        if (k + 1 < n) nxt = ld(idx(k + 1));
        double fx, fy, fz;
        if (pair_force(pa.x, pa.y, pa.z, pa.w, cur.x, cur.y, cur.z, cur.w, K, fx, fy, fz)) {
            Fx = Fx + fx;
            Fy = Fy + fy;
            Fz = Fz + fz;
        }
        cur = nxt;
    }
}

// The item (root or image) a lane's walk is in: its atom and entry range.
struct Item {
    uint64_t atom;
    uint32_t end;  // one past its last entry
};

// Item j of root t's group (0: t itself; j >= 1: its j-th image in fold
// order), starting at entry `begin`.
__device__ __forceinline__ Item item_at(const ForceSeq& p, uint64_t t, uint32_t f0, int j,
                                        uint32_t begin) {
    Item it;
    it.atom = j == 0 ? t : p.nlocal + p.fold_list[f0 + j - 1];
    it.end = begin + p.cnt[it.atom];
    return it;
}

// One warp tile of the grouped consumer: roots [32 w, 32 w + 32) and their
// images.  Phase 1 spreads the tile's entries over the lanes, U rows of 32 per
// chunk, and writes every pair force to shared memory; phase 2 lets each lane
// add its own group's entries of the chunk in order.  With FOLD, each lane
// then folds its images into its root (fold_root: reverse_send_force's order).
template <int U, bool FOLD>
__device__ __forceinline__ void force_tile(const ForceSeq& p, const AtomCols& c,
                                           const PlaneList& rev, uint64_t w, ForceSmem<U>& sm,
                                           int lane, int wib) {
    constexpr int CH = 32 * U;
    const uint64_t nl = p.nlocal;
    const uint64_t t = w * 32 + lane;
    const bool valid = t < nl;
    const uint64_t last = w * 32 + 32 < nl ? w * 32 + 32 : nl;
    double xa = 0.0, ya = 0.0, za = 0.0, ra = 0.0;
    uint32_t gs = 0, ge = 0, f0 = 0, nimg = 0;
    if (valid) {
        xa = c.x[t];
        ya = c.y[t];
        za = c.z[t];
        ra = p.rad[t];
        gs = p.grp_start[t];
        ge = p.grp_start[t + 1];
        f0 = p.fold_start[t];
        nimg = p.fold_start[t + 1] - f0;
    }
    const uint32_t base = p.grp_start[w * 32];
    const uint32_t end = p.grp_start[last];
    // the lane's walk over its group: current item j and its running sum
    int j = 0;
    Item it = {t, gs};
    if (valid) it = item_at(p, t, f0, 0, gs);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    uint32_t k = gs;
    for (uint32_t c0 = base; c0 < end; c0 += CH) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t e = c0 + (uint32_t)(u * 32 + lane);
            const bool in = e < end;
            uint32_t o = 0, m = 0;
            if (in) {
                o = p.seq[e];
                m = p.owner[e];
            }
            const int ol = (int)(m & 31u);
            double xi = __shfl_sync(0xffffffffu, xa, ol);
            double yi = __shfl_sync(0xffffffffu, ya, ol);
            double zi = __shfl_sync(0xffffffffu, za, ol);
            double ri = __shfl_sync(0xffffffffu, ra, ol);
            const uint32_t of0 = __shfl_sync(0xffffffffu, f0, ol);
            if (m >> 5) {  // an image of lane ol's root
                const uint64_t g = nl + p.fold_list[of0 + (m >> 5) - 1];
                xi = c.x[g];
                yi = c.y[g];
                zi = c.z[g];
                ri = p.rad[g];
            }
            double fx = 0.0, fy = 0.0, fz = 0.0;
            bool hit = false;
            if (in)
                hit = pair_force(xi, yi, zi, ri, c.x[o], c.y[o], c.z[o], p.rad[o], p.K, fx, fy, fz);
            const unsigned mask = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) sm.hit[wib][u] = mask;
            sm.fx[wib][u * 32 + lane] = fx;
            sm.fy[wib][u * 32 + lane] = fy;
            sm.fz[wib][u * 32 + lane] = fz;
        }
        __syncwarp();
        // this lane's entries inside the chunk, in group order
        const uint32_t hi = ge < c0 + CH ? ge : c0 + CH;
        for (; k < hi; ++k) {
            // k < ge = the last item's end, so the walk never passes it
            while (k >= it.end) {  // the item is complete: store its force
                c.fx[it.atom] = Fx;
                c.fy[it.atom] = Fy;
                c.fz[it.atom] = Fz;
                Fx = Fy = Fz = 0.0;
                ++j;
                it = item_at(p, t, f0, j, it.end);
            }
            const uint32_t r = k - c0;
            if (sm.hit[wib][r >> 5] & (1u << (r & 31))) {
                Fx = Fx + sm.fx[wib][r];
                Fy = Fy + sm.fy[wib][r];
                Fz = Fz + sm.fz[wib][r];
            }
        }
        __syncwarp();
    }
    if (valid) {
        // every entry is summed: store the open item, then the images after
        // it, which have no entries (their force is zero)
        for (;;) {
            c.fx[it.atom] = Fx;
            c.fy[it.atom] = Fy;
            c.fz[it.atom] = Fz;
            if (j == (int)nimg) break;
            Fx = Fy = Fz = 0.0;
            ++j;
            it = item_at(p, t, f0, j, it.end);
        }
        if (FOLD) fold_root(c, nl, t, p.fold_start, p.fold_list, rev);
    }
}

// Partner k of atom a's flattened order: in-list rows below a (npre of
// them), a's own row, the rest of the in-list.
struct CsrIdx {
    const uint32_t* in_list;
    const uint32_t* indices;
    uint32_t qs, npre, rs, nrow;
    __device__ __forceinline__ uint32_t operator()(uint32_t k) const {
        return k < npre ? in_list[qs + k]
             : k < npre + nrow ? indices[rs + (k - npre)] : in_list[qs + (k - nrow)];
    }
};

// The force on atom a (a root, or one of its ghost images) in the
// reference's summation order, from the transposed list and the CSR: in-list
// rows below a (ascending; in_split[a] of them), a's own row, the in-list
// rows above a; each entry evaluated as f(a, partner) (the negation argument
// at the top of k_force.cu).  Ghosts receive only with newton and have no row.
template <class Ld>
__device__ __forceinline__ void csr_item_force(const ForceCsr& q, const Ld& ld, uint64_t a,
                                               double& Fx, double& Fy, double& Fz) {
    const bool local = a < q.nlocal;
    const double4 pa = ld(a);
    Fx = 0.0;
    Fy = 0.0;
    Fz = 0.0;
    CsrIdx ix{q.in_list, q.indices, 0, 0, 0, 0};
    uint32_t nin = 0;
    if (q.newton || local) {
        ix.qs = q.in_start[a];
        nin = q.in_start[a + 1] - ix.qs;
        ix.npre = q.in_split[a];
    }
    if (local) {
        ix.rs = q.offsets[a];
        ix.nrow = q.offsets[a + 1] - ix.rs;
    }
    sum_partners(ld, pa, q.K, nin + ix.nrow, ix, Fx, Fy, Fz);
}

// Root t and its images by one thread (CSR walk), then (FOLD) the fold.
template <bool FOLD, class Ld>
__device__ __forceinline__ void force_csr_root_ld(const ForceCsr& q, const Ld& ld,
                                                  const AtomCols& c, const PlaneList& rev,
                                                  uint64_t t) {
    const uint32_t f0 = q.fold_start[t], f1 = q.fold_start[t + 1];
    for (uint32_t f = f0 - 1; f + 1 <= f1; ++f) {  // the root (f = f0 - 1), then its images
        const uint64_t a = f + 1 == f0 ? t : q.nlocal + q.fold_list[f];
        double Fx, Fy, Fz;
        csr_item_force(q, ld, a, Fx, Fy, Fz);
        c.fx[a] = Fx;
        c.fy[a] = Fy;
        c.fz[a] = Fz;
    }
    if (FOLD) fold_root(c, q.nlocal, t, q.fold_start, q.fold_list, rev);
}

// PK: the partners' records from q.pk (which must then be set), else from
// the columns.
template <bool FOLD, bool PK>
__device__ __forceinline__ void force_csr_root(const ForceCsr& q, const AtomCols& c,
                                               const PlaneList& rev, uint64_t t) {
    if constexpr (PK) force_csr_root_ld<FOLD>(q, PkLd{q.pk}, c, rev, t);
    else force_csr_root_ld<FOLD>(q, ColLd{c.x, c.y, c.z, q.rad}, c, rev, t);
}

// Entry k of a group's sequence.
struct SeqIdx {
    const uint32_t* seq;
    __device__ __forceinline__ uint32_t operator()(uint32_t k) const { return seq[k]; }
};

// Root t's group walked by one thread: each item's (root's, then every
// image's) sequence summed in order, its force written, then (FOLD) the
// images folded into the root in reverse_send_force's order.
template <bool FOLD, class Ld>
__device__ __forceinline__ void force_walk_root_ld(const ForceSeq& p, const Ld& ld,
                                                   const AtomCols& c, const PlaneList& rev,
                                                   uint64_t t) {
    const uint64_t nl = p.nlocal;
    const uint32_t f0 = p.fold_start[t], nimg = p.fold_start[t + 1] - f0;
    uint32_t k = p.grp_start[t];
    for (uint32_t j = 0; j <= nimg; ++j) {
        const uint64_t a = j == 0 ? t : nl + p.fold_list[f0 + j - 1];
        const uint32_t n = p.cnt[a];
        double Fx = 0.0, Fy = 0.0, Fz = 0.0;
        sum_partners(ld, ld(a), p.K, n, SeqIdx{p.seq + k}, Fx, Fy, Fz);
        k += n;
        c.fx[a] = Fx;
        c.fy[a] = Fy;
        c.fz[a] = Fz;
    }
    if (FOLD) fold_root(c, nl, t, p.fold_start, p.fold_list, rev);
}

template <bool FOLD, bool PK>
__device__ __forceinline__ void force_walk_root(const ForceSeq& p, const AtomCols& c,
                                                const PlaneList& rev, uint64_t t) {
    if constexpr (PK) force_walk_root_ld<FOLD>(p, PkLd{p.pk}, c, rev, t);
    else force_walk_root_ld<FOLD>(p, ColLd{c.x, c.y, c.z, p.rad}, c, rev, t);
}

}  // namespace soil
