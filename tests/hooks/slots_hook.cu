// slots_hook.cu — external consumers that keep per-contact history in the
// persistent neighbor slots (include/soil_slots.cuh).  Built by the GPU tests
// with -fmad=false; test code, not part of the library.
//
// contact_history_hook: the harmonic force through soil_gather_force (the
// built-in consumer's trajectory, bit for bit), plus, for every contact of a
// row atom i with partner j (overlap > 0, the force's own test), a 5-wide
// state: [steps in contact, sum of overlaps, sum of dx, dy, dz] with
// d = x_j - x_i.  The d sums depend on orientation: a state found in the
// partner's slots (the pair changed rows) is negated before use.
//
// self_count_hook: every local atom keeps one slot keyed by its own tag and
// adds 1 per step (the reference's own persistence test, through sorts).
#include <cuda_runtime.h>

#include "soil_consumer.cuh"
#include "soil_slots.cuh"

namespace {

__global__ void gather_forces(soil_dev_view v, double K) {
    const soil_harmonic_pair pair{v.x, v.y, v.z, v.columns[0], K};
    const uint64_t n = v.nlocal + v.nghost;
    for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n;
         a += (uint64_t)gridDim.x * blockDim.x) {
        double F[3];
        soil_gather_force(v, a, pair, F);
        v.fx[a] = F[0];
        v.fy[a] = F[1];
        v.fz[a] = F[2];
    }
}

__global__ void contact_history(soil_dev_view v, unsigned* overflow) {
    const double* rad = v.columns[0];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < v.nlocal;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t k = 0;
        for (uint32_t e = v.neighbor_offsets[i]; e < v.neighbor_offsets[i + 1]; ++e) {
            const uint32_t j = v.neighbor_indices[e];
            const double sum_r = rad[i] + rad[j];
            const double dx = v.x[j] - v.x[i];
            const double dy = v.y[j] - v.y[i];
            const double dz = v.z[j] - v.z[i];
            const double dist_sq = dx * dx + dy * dy + dz * dz;
            if (dist_sq >= sum_r * sum_r || dist_sq == 0.0) continue;
            const double overlap = sum_r - sqrt(dist_sq);
            double s[5];
            if (soil_slot_find(v, i, j, s) < 0) {
                s[2] = -s[2];
                s[3] = -s[3];
                s[4] = -s[4];
            }
            s[0] = s[0] + 1.0;
            s[1] = s[1] + overlap;
            s[2] = s[2] + dx;
            s[3] = s[3] + dy;
            s[4] = s[4] + dz;
            if (k < v.slot_max)
                soil_slot_put(v, i, k++, v.tag[j], s);
            else
                atomicAdd(overflow, 1u);
        }
        soil_slot_clear_from(v, i, k);
    }
}

__global__ void self_count(soil_dev_view v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < v.nlocal;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double s[8];
        soil_slot_find(v, i, i, s);
        s[0] = s[0] + 1.0;
        soil_slot_put(v, i, 0, v.tag[i], s);
        soil_slot_clear_from(v, i, 1);
    }
}

}  // namespace

struct history_user {
    double K;
    unsigned* overflow;  // device counter of contacts beyond slot_max
};

// user: pointer to a history_user
extern "C" int contact_history_hook(const soil_dev_view* v, void* user) {
    const history_user* u = static_cast<const history_user*>(user);
    if (!v->in_start || !v->in_list || v->slot_max == 0 || v->slot_width != 5) return 2;
    cudaStream_t st = static_cast<cudaStream_t>(v->stream);
    gather_forces<<<592, 256, 0, st>>>(*v, u->K);
    contact_history<<<592, 128, 0, st>>>(*v, u->overflow);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// user: pointer to the spring constant K (a double)
extern "C" int self_count_hook(const soil_dev_view* v, void* user) {
    if (!v->in_start || !v->in_list || v->slot_max == 0 || v->slot_width > 8) return 2;
    cudaStream_t st = static_cast<cudaStream_t>(v->stream);
    gather_forces<<<592, 256, 0, st>>>(*v, *static_cast<const double*>(user));
    self_count<<<592, 128, 0, st>>>(*v);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
