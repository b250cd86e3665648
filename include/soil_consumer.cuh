/* soil_consumer.cuh — device helpers for force consumers plugged in through
 * soil_sys_set_force_hook (header-only CUDA C++; include it from the
 * consumer's own .cu file).
 *
 * A reference consumer loops over pairs(nlocal) in CSR order and adds +f to
 * the row atom i and -f to j (the tutorial's soft_repulsion_force,
 * docs/src/tutorial/write-your-own-physics.md:56-110).  Atom a therefore
 * receives, in this order: -f(i, a) from every earlier row i that lists a
 * (ascending i), +f(a, j) over its own row, -f(i, a) from later rows; with
 * newton off a ghost receives nothing.  soil_gather_force walks exactly that
 * sequence for one atom from the view's CSR and its transpose, so one thread
 * per atom reproduces the reference's sums bit for bit with no atomics, for
 * any pair function.  f(i, j) is always evaluated with i the row atom, so both
 * atoms of a pair see the same value.  Compile consumers that must match the
 * reference's bits with -fmad=false (the reference never contracts a*b+c).
 *
 * soil_step folds ghost forces into their owners (reverse comm) after the
 * hook returns; the view's fold fields describe that program for reading
 * only. */
#ifndef SOIL_CONSUMER_CUH
#define SOIL_CONSUMER_CUH

#include <stdint.h>

#include "soil_cuda.h"

/* pair(i, j, f): writes the force on row atom i from pair (i, j) into f[3]
 * and returns true, or returns false when the pair does not interact. */
template <class Pair>
__device__ __forceinline__ void soil_gather_force(const soil_dev_view& v, uint64_t a,
                                                  const Pair& pair, double F[3]) {
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    const bool local = a < v.nlocal;
    const bool receives = v.newton || local;
    const uint32_t qs = v.in_start[a];
    const uint32_t nin = receives ? v.in_start[a + 1] - qs : 0u;
    const uint32_t rs = local ? v.neighbor_offsets[a] : 0u;
    const uint32_t nrow = local ? v.neighbor_offsets[a + 1] - rs : 0u;
    uint32_t npre = 0;  /* in-list rows below a (ascending, never a itself) */
    while (npre < nin && v.in_list[qs + npre] < (uint32_t)a) ++npre;
    const uint32_t total = nin + nrow;
    for (uint32_t k = 0; k < total; ++k) {
        const bool own = k >= npre && k < npre + nrow;
        const uint32_t o =
            own ? v.neighbor_indices[rs + (k - npre)] : v.in_list[qs + (k < npre ? k : k - nrow)];
        double f[3];
        if (own) {
            if (!pair((uint32_t)a, o, f)) continue;
            Fx = Fx + f[0];
            Fy = Fy + f[1];
            Fz = Fz + f[2];
        } else {
            if (!pair(o, (uint32_t)a, f)) continue;
            Fx = Fx - f[0];
            Fy = Fy - f[1];
            Fz = Fz - f[2];
        }
    }
    F[0] = Fx;
    F[1] = Fy;
    F[2] = Fz;
}

/* The tutorial's linear repulsion as a pair function: d = x_j - x_i,
 * overlap = (r_i + r_j) - |d|, f_i = -K * overlap * d / |d| (operation for
 * operation as the built-in consumer). */
struct soil_harmonic_pair {
    const double* x;
    const double* y;
    const double* z;
    const double* radius;
    double K;
    __device__ __forceinline__ bool operator()(uint32_t i, uint32_t j, double f[3]) const {
        const double sum_r = radius[i] + radius[j];
        const double dx = x[j] - x[i];
        const double dy = y[j] - y[i];
        const double dz = z[j] - z[i];
        const double dist_sq = dx * dx + dy * dy + dz * dz;
        if (dist_sq >= sum_r * sum_r || dist_sq == 0.0) return false;
        const double dist = sqrt(dist_sq);
        const double overlap = sum_r - dist;
        const double inv_dist = 1.0 / dist;
        const double fmag = K * overlap;
        f[0] = -fmag * dx * inv_dist;
        f[1] = -fmag * dy * inv_dist;
        f[2] = -fmag * dz * inv_dist;
        return true;
    }
};

#endif /* SOIL_CONSUMER_CUH */
