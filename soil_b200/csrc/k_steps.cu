// k_steps.cu — device-resident communicate-only steps.
//
// The reference decides every step whether the lists must be rebuilt
// (decide_rebuild, crates/soil_core/src/neighbor.rs:796-822); its GPU
// prototype runs K resident steps with no host read in between
// (crates/soil_gpu/src/gpu_state.rs:352-418).  k_steps runs consecutive steps
// that keep their lists in ONE cooperative launch, every CTA resident:
//
//   phase A  final(t-1) + initial(t) + displacement check + forward comm
//            (the fused integration pass of soil_step), one thread per local;
//   barrier; every CTA reads the check: if any atom moved too far, the
//            launch ends here (step t's integration is done, its rebuild is
//            the host's);
//   phase B  the grouped consumer with the reverse fold (if any), then a
//            barrier (the next phase A reads the forces and moves the atoms
//            phase B reads); next step.  Without a consumer one barrier per
//            step suffices: the check flag rotates through three slots, so a
//            slot is cleared only after every CTA has read it.
//
// Each step runs the same per-atom functions in the same order as the
// launch-per-phase path, so results are bit-identical.  The grid barrier is
// this library's own (a counter and a generation word): its wait is bounded,
// and a CTA whose wait runs out records SOIL_STEPS_ERR_BARRIER in flags->error
// and returns; the others then run out at their next barrier.  Co-residency
// of every CTA is guaranteed by the cooperative launch, so the bound is a
// guard, never the expected exit.
#include <cuda/atomic>

#include "device_ops.cuh"
#include "force_ops.cuh"
#include "kernels.cuh"

namespace soil {

namespace {

// Spins of a barrier wait (each >= 100 ns of __nanosleep): about a second.
constexpr uint64_t kBarrierSpinLimit = 1ull << 23;

// Grid barrier.  *watch (when given) is read by thread 0 after the barrier
// and returned to every thread of the CTA in *seen (one load per CTA, not
// one per thread, of a word every CTA polls).
__device__ bool grid_sync(GridBar* b, unsigned nblocks, unsigned& gen, uint32_t* err,
                          const uint32_t* watch = nullptr, uint32_t* seen = nullptr) {
    __shared__ int ok;
    __shared__ uint32_t s_seen;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(b->count), g(b->gen);
        ok = 1;
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            g.store(gen + 1, cuda::memory_order_release);
        } else {
            uint64_t spins = 0;
            while (g.load(cuda::memory_order_acquire) == gen) {
                if (++spins > kBarrierSpinLimit) {
                    atomicOr(err, SOIL_STEPS_ERR_BARRIER);
                    ok = 0;
                    break;
                }
                if (spins > 256) __nanosleep(100);  // a short busy wait first
            }
        }
        gen += 1;
        if (watch)
            s_seen = cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(
                         *const_cast<uint32_t*>(watch))
                         .load(cuda::memory_order_relaxed);
    }
    __syncthreads();
    if (seen) *seen = s_seen;
    return ok != 0;
}

}  // namespace

// CONSUMER: 0 none, 1 without fold, 2 with fold (newton).  MODE: 0 warp
// tiles over grouped sequences (force_tile), 1 one root per thread over
// them (force_walk_root), 2 one root per thread over the CSR and its
// transpose (force_csr_root).
template <int U, int CONSUMER, int MODE, bool PK>
__global__ void __launch_bounds__(kBlock, 4) k_steps(StepsArgs a) {
    __shared__ ForceSmem<U> sm;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint64_t nl = a.nlocal;
    const AtomCols& c = a.c;
    // every CTA reads the generation before any CTA can reach the first
    // barrier's release (which needs all of them)
    unsigned gen = 0;
    if (threadIdx.x == 0)
        gen = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(a.bar->gen)
                  .load(cuda::memory_order_relaxed);
    uint64_t done = 0;
    bool stop = false;
    for (uint64_t step = 0; step < a.max_steps; ++step) {
        // the check flag of this step: three slots in rotation, so a slot is
        // cleared (two steps ahead, by CTA 0) only after every CTA read it
        uint32_t* slot = a.trip + step % 3;
        // phase A: the fused integration pass
        const bool fuse_final = step > 0 || a.first_fused;
        bool hit = false;
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nl;
             i += (uint64_t)gridDim.x * blockDim.x) {
            const double lx = a.ck.lbx[i], ly = a.ck.lby[i], lz = a.ck.lbz[i];  // before the stores
            double x, y, z, vx, vy, vz;
            initial_atom(c, i, a.dt, fuse_final, a.zero_force != 0, x, y, z, vx, vy, vz);
            hit |= check_moved_at(a.ck, x, y, z, lx, ly, lz);
            forward_images(c, nl, i, x, y, z, vx, vy, vz, a.fw.fold_start, a.fw.fold_list,
                           a.fw.chain, a.fw.sc, a.fw.fwd, a.fw.zero_ghost_force != 0);
        }
        if (__ballot_sync(0xffffffffu, hit) && lane == 0) atomicOr(slot, 1u);
        uint32_t tripped = 0;
        if (!grid_sync(a.bar, gridDim.x, gen, &a.flags->error, slot, &tripped)) return;
        if (tripped) {
            stop = true;
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0)
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(a.trip[(step + 2) % 3])
                .store(0u, cuda::memory_order_relaxed);
        // phase B: the consumer over every root's group (and the fold)
        if (CONSUMER && MODE == 2) {  // whole blocks of roots, in their order
            for (uint64_t b = (uint64_t)blockIdx.x * kBlock; b < nl;
                 b += (uint64_t)gridDim.x * kBlock) {
                const uint64_t k = b + threadIdx.x;
                if (k < nl)
                    force_csr_root<CONSUMER == 2, PK>(a.fc, c, a.fa.rev,
                                                      a.fc.order ? a.fc.order[k] : k);
            }
        } else if (CONSUMER && MODE == 1) {
            for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nl;
                 t += (uint64_t)gridDim.x * blockDim.x)
                force_walk_root<CONSUMER == 2, PK>(a.fa.q, c, a.fa.rev, t);
        } else if (CONSUMER) {
            const uint64_t ntiles = (nl + 31) / 32;
            for (uint64_t w = (uint64_t)blockIdx.x * kForceWarps + wib; w < ntiles;
                 w += (uint64_t)gridDim.x * kForceWarps)
                force_tile<U, CONSUMER == 2>(a.fa.q, c, a.fa.rev, w, sm, lane, wib);
        }
        // phase A of the next step reads the forces and moves the atoms
        // phase B reads: with a consumer, every CTA must be done first
        if (CONSUMER && !grid_sync(a.bar, gridDim.x, gen, &a.flags->error)) return;
        ++done;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = (uint32_t)done;
        a.out[1] = stop ? 1u : 0u;
        if (stop) a.flags->rebuild = 1u;  // decide_rebuild on the host reads it
    }
}

// PK (modes 1 and 2): the walks read the packed records.
static const void* steps_kernel(int consumer, int mode, bool pk) {
    if (consumer == 0) return (const void*)k_steps<4, 0, 2, false>;
    if (mode == 2) {
        if (pk)
            return consumer == 1 ? (const void*)k_steps<4, 1, 2, true>
                                 : (const void*)k_steps<4, 2, 2, true>;
        return consumer == 1 ? (const void*)k_steps<4, 1, 2, false>
                             : (const void*)k_steps<4, 2, 2, false>;
    }
    if (mode == 1) {
        if (pk)
            return consumer == 1 ? (const void*)k_steps<4, 1, 1, true>
                                 : (const void*)k_steps<4, 2, 1, true>;
        return consumer == 1 ? (const void*)k_steps<4, 1, 1, false>
                             : (const void*)k_steps<4, 2, 1, false>;
    }
    return consumer == 1 ? (const void*)k_steps<4, 1, 0, false> : (const void*)k_steps<4, 2, 0, false>;
}

int steps_grid(int consumer, int walk, bool pk, uint64_t nlocal, int* grid) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, steps_kernel(consumer, walk, pk), kBlock,
                                                      0) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return 1;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t need_atoms = (nlocal + kBlock - 1) / kBlock;
    const uint64_t need_tiles = ((nlocal + 31) / 32 + kForceWarps - 1) / kForceWarps;
    uint64_t need = need_atoms > need_tiles ? need_atoms : need_tiles;
    if (need < 1) need = 1;
    // one CTA per kBlock atoms (capped at residency): fewer CTAs striding over
    // more atoms each measured slower (32 CTAs: 19.6 vs 13.2 us per light step
    // on 32,768 atoms)
    const uint64_t cap = (uint64_t)per_sm * (uint64_t)sms;
    *grid = (int)(need < cap ? need : cap);
    return 0;
}

cudaError_t launch_steps(cudaStream_t st, const StepsArgs& a, int consumer, int walk, bool pk,
                         int grid) {
    note_launch();
    StepsArgs arg = a;
    void* params[] = {&arg};
    return cudaLaunchCooperativeKernel(steps_kernel(consumer, walk, pk), dim3(grid), dim3(kBlock),
                                       params, 0, st);
}

}  // namespace soil
