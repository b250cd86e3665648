// k_integrate.cu — velocity-Verlet half-steps, force zeroing, periodic wrap,
// the shear streaming profile and the build-position snapshot.
//
// All of these are HBM-bound streams over SoA f64 columns (0.1 flop/byte):
// one thread per atom, grid-stride, coalesced 8-byte accesses.
#include <cstdlib>
#include <atomic>

#include "device_ops.cuh"
#include "kernels.cuh"

namespace soil {

static std::atomic<uint64_t> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
bool pdl_on() {
    static const bool on = [] {
        const char* env = std::getenv("SOIL_PDL");
        return !(env && std::atoi(env) == 0);
    }();
    return on;
}
uint64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

unsigned grid_for(uint64_t n, int block, int per_sm) {
    uint64_t need = (n + block - 1) / block;
    uint64_t cap = 148ull * per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

// initial_integration, soil_verlet/src/lib.rs:131-162:
//   h = 0.5*dt*inv_m;  v += h*F;  x += v*dt
// With FWD, each local then writes its ghost images (forward_comm of a step
// that keeps its lists): the values forward comm would copy after this pass.
// Capped at 48 registers (5 blocks per SM) without spills.
template <bool FUSE_FINAL, bool FWD>
__global__ void __launch_bounds__(kBlock, 5) k_initial(uint64_t n, AtomCols c, double dt,
                                                    int zero_force, CheckArgs ck, FwdArgs fw) {
    pdl_wait();  // launched with pdl_launch
    bool hit = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const bool chk = i < ck.n_check;
        double lx = 0.0, ly = 0.0, lz = 0.0;  // build positions, loaded before the pass's stores
        if (chk) {
            lx = ck.lbx[i];
            ly = ck.lby[i];
            lz = ck.lbz[i];
        }
        double x, y, z, vx, vy, vz;
        initial_atom(c, i, dt, FUSE_FINAL, zero_force != 0, x, y, z, vx, vy, vz);
        if (chk) hit |= check_moved_at(ck, x, y, z, lx, ly, lz);
        if (FWD)
            forward_images(c, n, i, x, y, z, vx, vy, vz, fw.fold_start, fw.fold_list, fw.chain,
                           fw.sc, fw.fwd, fw.zero_ghost_force != 0);
    }
    if (ck.flags) {
        unsigned any = __ballot_sync(0xffffffffu, hit);
        if (any && (threadIdx.x & 31) == 0) atomicOr(&ck.flags->rebuild, 1u);
    }
}

CheckArgs make_check(const double* lbx, const double* lby, const double* lbz,
                            uint64_t n_check, double thr_sq, const double box[3],
                            DevFlags* flags, int mask) {
    CheckArgs ck;
    ck.mask = mask;
    ck.lbx = lbx;
    ck.lby = lby;
    ck.lbz = lbz;
    ck.n_check = lbx ? n_check : 0;
    ck.thr_sq = thr_sq;
    for (int d = 0; d < 3; ++d) {
        ck.box[d] = box ? box[d] : 1.0;
        ck.ibox[d] = 1.0 / ck.box[d];  // ibx = 1.0 / bx (neighbor.rs:716-718)
    }
    ck.flags = lbx ? flags : nullptr;
    return ck;
}

template <bool FUSE_FINAL>
static void initial_kernel(cudaStream_t st, uint64_t n, const AtomCols& c, double dt,
                           bool zero_force, const CheckArgs& ck, const FwdArgs* fw) {
    note_launch();
    if (fw) {
        pdl_launch(k_initial<FUSE_FINAL, true>, grid_wave<k_initial<FUSE_FINAL, true>>(n), kBlock, 0, st, 
            n, c, dt, zero_force ? 1 : 0, ck, *fw);
    } else {
        FwdArgs none{};
        pdl_launch(k_initial<FUSE_FINAL, false>, grid_wave<k_initial<FUSE_FINAL, false>>(n), kBlock, 0, st, 
            n, c, dt, zero_force ? 1 : 0, ck, none);
    }
}

void launch_initial(cudaStream_t st, uint64_t n, const AtomCols& c, double dt, bool zero_force,
                    const double* lbx, const double* lby, const double* lbz, uint64_t n_check,
                    double thr_sq, const double box[3], DevFlags* flags, int pbc_mask,
                    const FwdArgs* fw) {
    if (n == 0) return;
    CheckArgs ck = make_check(lbx, lby, lbz, n_check, thr_sq, box, flags, pbc_mask);
    initial_kernel<false>(st, n, c, dt, zero_force, ck, fw);
}

void launch_final_initial(cudaStream_t st, uint64_t n, const AtomCols& c, double dt,
                          bool zero_force, const double* lbx, const double* lby,
                          const double* lbz, uint64_t n_check, double thr_sq,
                          const double box[3], DevFlags* flags, int pbc_mask, const FwdArgs* fw) {
    if (n == 0) return;
    CheckArgs ck = make_check(lbx, lby, lbz, n_check, thr_sq, box, flags, pbc_mask);
    initial_kernel<true>(st, n, c, dt, zero_force, ck, fw);
}

// final_integration, soil_verlet/src/lib.rs:175-194: v += h*F
__global__ void __launch_bounds__(kBlock) k_final(uint64_t n, AtomCols c, double dt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        final_atom(c, i, dt);
}

void launch_final(cudaStream_t st, uint64_t n, const AtomCols& c, double dt) {
    if (n == 0) return;
    note_launch();
    k_final<<<grid_wave<k_final>(n), kBlock, 0, st>>>(n, c, dt);
}

__global__ void __launch_bounds__(kBlock) k_zero(uint64_t n, AtomCols c, PlaneList zp) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        c.fx[i] = 0.0;
        c.fy[i] = 0.0;
        c.fz[i] = 0.0;
        for (int k = 0; k < zp.n; ++k) c.planes[zp.idx[k]][i] = 0.0;
    }
}

void launch_zero_forces(cudaStream_t st, uint64_t n, const AtomCols& c, const int* zero_planes,
                        int nzero) {
    if (n == 0) return;
    PlaneList zp;
    zp.n = nzero;
    for (int k = 0; k < nzero; ++k) zp.idx[k] = zero_planes[k];
    note_launch();
    k_zero<<<grid_wave<k_zero>(n), kBlock, 0, st>>>(n, c, zp);
}

// pbc fully periodic fast path (domain.rs:626-636) / pbc_triclinic (domain.rs:674-729)
__global__ void __launch_bounds__(kBlock) k_pbc(uint64_t n, AtomCols c, Geom g, double bv0,
                                                double bv1, double bv2) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        pbc_atom(c, i, g, bv0, bv1, bv2);
}

void launch_pbc(cudaStream_t st, uint64_t nlocal, const AtomCols& c, const Geom& g,
                const double bvel[3]) {
    if (nlocal == 0) return;
    note_launch();
    k_pbc<<<grid_wave<k_pbc>(nlocal), kBlock, 0, st>>>(nlocal, c, g, bvel[0], bvel[1], bvel[2]);
}

// soil_deform/src/lib.rs:568-574: vel.x += rate*(y - yc) on the first shear step
__global__ void __launch_bounds__(kBlock) k_shear_profile(uint64_t n, AtomCols c, double rate,
                                                          double yc) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        c.vx[i] = c.vx[i] + rate * (c.y[i] - yc);
}

void launch_shear_profile(cudaStream_t st, uint64_t n, const AtomCols& c, double rate, double yc) {
    if (n == 0) return;
    note_launch();
    k_shear_profile<<<grid_wave<k_shear_profile>(n), kBlock, 0, st>>>(n, c, rate, yc);
}

// apply_deform's remap (soil_deform/src/lib.rs:530-540), one dim after another
__global__ void __launch_bounds__(kBlock) k_remap(uint64_t n, AtomCols c, RemapSpec r) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
    {
        for (int q = 0; q < r.n; ++q) {
            double* x = r.dim[q] == 0 ? c.x : r.dim[q] == 1 ? c.y : c.z;
            x[i] = r.new_center[q] + (x[i] - r.old_center[q]) * r.scale[q];
        }
        if (c.pk) put_pk(c.pk, i, c.x[i], c.y[i], c.z[i], c.pkrad[i]);
    }
}

void launch_remap(cudaStream_t st, uint64_t n, const AtomCols& c, const RemapSpec& r) {
    if (n == 0 || r.n == 0) return;
    note_launch();
    k_remap<<<grid_wave<k_remap>(n), kBlock, 0, st>>>(n, c, r);
}

}  // namespace soil

namespace soil {

// displacement_exceeded as a standalone pass (per-phase API path)
__global__ void __launch_bounds__(kBlock) k_disp_check(uint64_t n, AtomCols c, CheckArgs ck) {
    bool hit = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        hit |= check_moved(ck, c.x[i], c.y[i], c.z[i], i);
    if (__ballot_sync(0xffffffffu, hit) && (threadIdx.x & 31) == 0)
        atomicOr(&ck.flags->rebuild, 1u);
}

void launch_disp_check(cudaStream_t st, uint64_t n, const AtomCols& c, const double* lbx,
                       const double* lby, const double* lbz, double thr_sq, const double box[3],
                       DevFlags* flags, int pbc_mask) {
    if (n == 0) return;
    CheckArgs ck = make_check(lbx, lby, lbz, n, thr_sq, box, flags, pbc_mask);
    note_launch();
    k_disp_check<<<grid_wave<k_disp_check>(n), kBlock, 0, st>>>(n, c, ck);
}

// [n][3] interleaved <-> three SoA planes (host-facing layout of Vec<[f64;3]>)
__global__ void __launch_bounds__(kBlock) k_deinterleave3(uint64_t n, const double* src, double* a,
                                                          double* b, double* c) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        a[i] = src[3 * i];
        b[i] = src[3 * i + 1];
        c[i] = src[3 * i + 2];
    }
}
__global__ void __launch_bounds__(kBlock) k_interleave3(uint64_t n, double* dst, const double* a,
                                                        const double* b, const double* c) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        dst[3 * i] = a[i];
        dst[3 * i + 1] = b[i];
        dst[3 * i + 2] = c[i];
    }
}
__global__ void __launch_bounds__(kBlock) k_interleave3i(uint64_t n, int32_t* dst, const int32_t* a,
                                                         const int32_t* b, const int32_t* c) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        dst[3 * i] = a[i];
        dst[3 * i + 1] = b[i];
        dst[3 * i + 2] = c[i];
    }
}
// column of width w: [n][w] interleaved <-> w planes of stride cap
__global__ void __launch_bounds__(kBlock) k_deinterleave_w(uint64_t n, int w, const double* src,
                                                           double* dst0, uint64_t cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < w; ++k) dst0[k * cap + i] = src[(uint64_t)w * i + k];
}
__global__ void __launch_bounds__(kBlock) k_interleave_w(uint64_t n, int w, double* dst,
                                                         const double* src0, uint64_t cap) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < w; ++k) dst[(uint64_t)w * i + k] = src0[k * cap + i];
}

void launch_deinterleave3(cudaStream_t st, uint64_t n, const double* src, double* a, double* b,
                          double* c) {
    if (n) {
        note_launch();
        k_deinterleave3<<<grid_wave<k_deinterleave3>(n), kBlock, 0, st>>>(n, src, a, b, c);
    }
}
void launch_interleave3(cudaStream_t st, uint64_t n, double* dst, const double* a, const double* b,
                        const double* c) {
    if (n) {
        note_launch();
        k_interleave3<<<grid_wave<k_interleave3>(n), kBlock, 0, st>>>(n, dst, a, b, c);
    }
}
void launch_interleave3i(cudaStream_t st, uint64_t n, int32_t* dst, const int32_t* a,
                         const int32_t* b, const int32_t* c) {
    if (n) {
        note_launch();
        k_interleave3i<<<grid_wave<k_interleave3i>(n), kBlock, 0, st>>>(n, dst, a, b, c);
    }
}
// inv[i] = 1.0 / m[i] (IEEE division, the host's bits)
__global__ void __launch_bounds__(kBlock) k_inverse(uint64_t n, const double* m, double* inv) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        inv[i] = 1.0 / m[i];
}
void launch_inverse(cudaStream_t st, uint64_t n, const double* m, double* inv) {
    if (n) {
        note_launch();
        k_inverse<<<grid_wave<k_inverse>(n), kBlock, 0, st>>>(n, m, inv);
    }
}

void launch_deinterleave_w(cudaStream_t st, uint64_t n, int w, const double* src, double* dst0,
                           uint64_t cap) {
    if (n) {
        note_launch();
        k_deinterleave_w<<<grid_wave<k_deinterleave_w>(n), kBlock, 0, st>>>(n, w, src, dst0, cap);
    }
}
void launch_interleave_w(cudaStream_t st, uint64_t n, int w, double* dst, const double* src0,
                         uint64_t cap) {
    if (n) {
        note_launch();
        k_interleave_w<<<grid_wave<k_interleave_w>(n), kBlock, 0, st>>>(n, w, dst, src0, cap);
    }
}

__global__ void __launch_bounds__(kBlock) k_pack(uint64_t n, AtomCols c, const double* rad,
                                                 double* pk) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        put_pk(pk, i, c.x[i], c.y[i], c.z[i], rad[i]);
    }
}

void launch_pack(cudaStream_t st, uint64_t n, const AtomCols& c, const double* rad, double* pk) {
    if (n == 0) return;
    note_launch();
    k_pack<<<grid_wave<k_pack>(n), kBlock, 0, st>>>(n, c, rad, pk);
}

}  // namespace soil
