// k_force.cu — the built-in pair consumer: linear repulsion
// f = k*overlap along the line of centres, the tutorial's
// soft_repulsion_force (docs/src/tutorial/write-your-own-physics.md:56-110).
//
// The reference accumulates pair forces in global pair order: for pair
// (i, j) it adds +f to i and -f to j, rows ascending, CSR order inside a row.
// So atom a receives, in order, -f(i,a) from every earlier row i that lists
// a (ascending i), then +f(a,j) for its own row, then (full lists only) -f
// from later rows.  This kernel gathers exactly that sequence per atom from
// the CSR and its transpose — one thread per atom, no atomics — so the sums
// are bit-identical to the sequential reference.  f(i,j) is always evaluated
// with i the row atom, so both endpoints recompute the same value.
#include "kernels.cuh"

namespace soil {

struct PairForce {
    bool hit;
    double fx, fy, fz;
};

__device__ __forceinline__ PairForce pair_force(const AtomCols& c, const double* rad, double K,
                                                uint32_t i, uint32_t j) {
    PairForce f;
    f.hit = false;
    const double ri = rad[i], rj = rad[j];
    const double sum_r = ri + rj;
    const double dx = c.x[j] - c.x[i];
    const double dy = c.y[j] - c.y[i];
    const double dz = c.z[j] - c.z[i];
    const double dist_sq = dx * dx + dy * dy + dz * dz;
    if (dist_sq >= sum_r * sum_r || dist_sq == 0.0) return f;
    const double dist = sqrt(dist_sq);
    const double overlap = sum_r - dist;
    const double inv_dist = 1.0 / dist;
    const double fmag = K * overlap;
    f.hit = true;
    f.fx = -fmag * dx * inv_dist;
    f.fy = -fmag * dy * inv_dist;
    f.fz = -fmag * dz * inv_dist;
    return f;
}

__global__ void __launch_bounds__(kBlock) k_harmonic(uint64_t nlocal, uint64_t ntotal, AtomCols c,
                                                     const double* rad, double K, int newton,
                                                     const uint32_t* offsets,
                                                     const uint32_t* indices,
                                                     const uint32_t* in_start,
                                                     const uint32_t* in_list) {
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < ntotal;
         a += (uint64_t)gridDim.x * blockDim.x) {
        double Fx = 0.0, Fy = 0.0, Fz = 0.0;
        const bool local = a < nlocal;
        // reference applies -f to j only when newton || j < nlocal
        const bool receives = newton || local;
        uint32_t q = in_start[a];
        const uint32_t qe = in_start[a + 1];
        if (receives) {
            for (; q < qe; ++q) {
                const uint32_t i = in_list[q];
                if (i > a) break;  // later rows come after this atom's own row
                const PairForce f = pair_force(c, rad, K, i, (uint32_t)a);
                if (f.hit) {
                    Fx = Fx - f.fx;
                    Fy = Fy - f.fy;
                    Fz = Fz - f.fz;
                }
            }
        }
        if (local) {
            for (uint32_t p = offsets[a]; p < offsets[a + 1]; ++p) {
                const PairForce f = pair_force(c, rad, K, (uint32_t)a, indices[p]);
                if (f.hit) {
                    Fx = Fx + f.fx;
                    Fy = Fy + f.fy;
                    Fz = Fz + f.fz;
                }
            }
        }
        if (receives) {
            for (; q < qe; ++q) {
                const uint32_t i = in_list[q];
                const PairForce f = pair_force(c, rad, K, i, (uint32_t)a);
                if (f.hit) {
                    Fx = Fx - f.fx;
                    Fy = Fy - f.fy;
                    Fz = Fz - f.fz;
                }
            }
        }
        c.fx[a] = Fx;
        c.fy[a] = Fy;
        c.fz[a] = Fz;
    }
}

void launch_harmonic(cudaStream_t st, uint64_t nlocal, uint64_t ntotal, const AtomCols& c,
                     const double* radius, double k, int newton, const uint32_t* offsets,
                     const uint32_t* indices, const uint32_t* in_start, const uint32_t* in_list) {
    if (ntotal == 0) return;
    note_launch();
    k_harmonic<<<grid_for(ntotal), kBlock, 0, st>>>(nlocal, ntotal, c, radius, k, newton, offsets,
                                                    indices, in_start, in_list);
}

}  // namespace soil
