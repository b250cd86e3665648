// k_ghost.cu — periodic / Lees–Edwards ghost images on one GPU.
//
// borders (comm.rs:682-860): for dim in x,y,z the lo swap (shift +L) then
// the hi swap (shift -L) scan the locals plus the ghosts of earlier dims in
// index order and append every atom inside the face slab.  The device version
// is an order-preserving stream compaction: per 2048-atom tile count the lo
// and hi selections, scan the tile counts, then each tile re-derives its
// flags, ranks them with a CTA scan and writes the ghosts at their final
// slots — so ghost order, send lists and recv ranges equal the reference's.
//
// forward_comm (comm.rs:400-432): the reference packs pos+offset from the
// source (a local or an earlier ghost) swap by swap.  Every ghost therefore
// equals its root local atom plus the offsets of its swap chain, added in
// chain order; borders records (root, chain) so one kernel refreshes all
// ghosts with the exact same additions.
//
// reverse_send_force (comm.rs:938-1024): swaps are folded last to first,
// lo before hi, F[send[k]] += F[recv_start+k]; one launch per swap keeps
// that order (targets inside a swap are distinct, so no atomics).
#include "block_scan.cuh"
#include "kernels.cuh"

namespace soil {

constexpr int kBorderItems = kBorderTile / kBlock;

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

__global__ void __launch_bounds__(kBlock) k_border_count(uint64_t scan_end, AtomCols c, BorderDim bd,
                                                         uint32_t* tile_lo, uint32_t* tile_hi) {
    __shared__ uint32_t tot;
    const uint64_t base = (uint64_t)blockIdx.x * kBorderTile + (uint64_t)threadIdx.x * kBorderItems;
    uint32_t nlo = 0, nhi = 0;
    for (int k = 0; k < kBorderItems; ++k) {
        const uint64_t i = base + k;
        if (i >= scan_end) break;
        bool lo, hi;
        border_flags(c, bd, i, lo, hi);
        nlo += lo;
        nhi += hi;
    }
    block_exclusive_scan(nlo, &tot);
    if (threadIdx.x == 0) tile_lo[blockIdx.x] = tot;
    block_exclusive_scan(nhi, &tot);
    if (threadIdx.x == 0) tile_hi[blockIdx.x] = tot;
}

void launch_border_count(cudaStream_t st, uint64_t scan_end, const AtomCols& c,
                         const BorderDim& bd, uint32_t* tile_lo, uint32_t* tile_hi) {
    const uint64_t tiles = (scan_end + kBorderTile - 1) / kBorderTile;
    if (tiles == 0) return;
    note_launch();
    k_border_count<<<(unsigned)tiles, kBlock, 0, st>>>(scan_end, c, bd, tile_lo, tile_hi);
}

// Ghost g := image of atom i through swap `s` (pack_border + unpack_atom,
// atom.rs:520-553; registry pack_all/unpack_all for every column).
__device__ __forceinline__ void write_ghost(const AtomCols& c, uint64_t g, uint64_t i,
                                            const double* shift, const double* vshift, int s,
                                            uint64_t nlocal, uint32_t* root, uint32_t* chain) {
    const uint64_t cap = c.cap;
    c.x[g] = c.x[i] + shift[0];
    c.y[g] = c.y[i] + shift[1];
    c.z[g] = c.z[i] + shift[2];
    c.vx[g] = c.vx[i] + vshift[0];
    c.vy[g] = c.vy[i] + vshift[1];
    c.vz[g] = c.vz[i] + vshift[2];
    c.fx[g] = c.fx[i];
    c.fy[g] = c.fy[i];
    c.fz[g] = c.fz[i];
    const double m = c.mass[i];
    c.mass[g] = m;
    c.inv_mass[g] = 1.0 / m;
    c.cut[g] = c.cut[i];
    c.tag[g] = c.tag[i];
    c.type[g] = c.type[i];
    c.img[g] = c.img[i];
    c.img[cap + g] = c.img[cap + i];
    c.img[2 * cap + g] = c.img[2 * cap + i];
    c.origin[g] = (int32_t)i;
    for (int q = 0; q < c.nplanes; ++q) c.planes[q][g] = c.planes[q][i];
    // chain: swap ids in 3-bit fields (application order), length in bits 12-13
    uint32_t r, code;
    if (i < nlocal) {
        r = (uint32_t)i;
        code = (1u << 12) | (uint32_t)s;
    } else {
        r = root[i - nlocal];
        const uint32_t pc = chain[i - nlocal];
        const uint32_t len = pc >> 12;
        code = (pc & 0xfffu) | ((uint32_t)s << (3 * len)) | ((len + 1) << 12);
    }
    root[g - nlocal] = r;
    chain[g - nlocal] = code;
}

__global__ void __launch_bounds__(kBlock) k_border_scatter(
    uint64_t scan_end, uint64_t nlocal, AtomCols c, BorderDim bd, const uint32_t* tile_off_lo,
    const uint32_t* tile_off_hi, uint64_t recv_lo, uint64_t recv_hi, uint32_t* send_lo,
    uint32_t* send_hi, uint32_t* root, uint32_t* chain) {
    __shared__ uint32_t tot;
    const uint64_t base = (uint64_t)blockIdx.x * kBorderTile + (uint64_t)threadIdx.x * kBorderItems;
    uint32_t flo = 0, fhi = 0;  // bit k: item k selected
    for (int k = 0; k < kBorderItems; ++k) {
        const uint64_t i = base + k;
        if (i >= scan_end) break;
        bool lo, hi;
        border_flags(c, bd, i, lo, hi);
        flo |= (uint32_t)lo << k;
        fhi |= (uint32_t)hi << k;
    }
    uint32_t rlo = block_exclusive_scan(__popc(flo), &tot) + tile_off_lo[blockIdx.x];
    uint32_t rhi = block_exclusive_scan(__popc(fhi), &tot) + tile_off_hi[blockIdx.x];
    for (int k = 0; k < kBorderItems; ++k) {
        const uint64_t i = base + k;
        if ((flo >> k) & 1u) {
            write_ghost(c, recv_lo + rlo, i, bd.shift[0], bd.vshift[0], bd.swap_id[0], nlocal, root,
                        chain);
            send_lo[rlo] = (uint32_t)i;
            ++rlo;
        }
        if ((fhi >> k) & 1u) {
            write_ghost(c, recv_hi + rhi, i, bd.shift[1], bd.vshift[1], bd.swap_id[1], nlocal, root,
                        chain);
            send_hi[rhi] = (uint32_t)i;
            ++rhi;
        }
    }
}

void launch_border_scatter(cudaStream_t st, uint64_t scan_end, uint64_t nlocal, const AtomCols& c,
                           const BorderDim& bd, const uint32_t* tile_off_lo,
                           const uint32_t* tile_off_hi, uint64_t recv_lo, uint64_t recv_hi,
                           uint32_t* send_lo, uint32_t* send_hi, uint32_t* ghost_root,
                           uint32_t* ghost_chain) {
    const uint64_t tiles = (scan_end + kBorderTile - 1) / kBorderTile;
    if (tiles == 0) return;
    note_launch();
    k_border_scatter<<<(unsigned)tiles, kBlock, 0, st>>>(scan_end, nlocal, c, bd, tile_off_lo,
                                                         tile_off_hi, recv_lo, recv_hi, send_lo,
                                                         send_hi, ghost_root, ghost_chain);
}

struct PlaneList {
    int idx[kMaxPlanes];
    int n;
};

__global__ void __launch_bounds__(kBlock) k_forward(uint64_t nlocal, uint64_t nghost, AtomCols c,
                                                    const uint32_t* root, const uint32_t* chain,
                                                    SwapConst sc, PlaneList fwd, int zero_force) {
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nghost;
         gi += (uint64_t)gridDim.x * blockDim.x) {
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
        if (zero_force) {
            c.fx[g] = 0.0;
            c.fy[g] = 0.0;
            c.fz[g] = 0.0;
        }
    }
}

void launch_forward(cudaStream_t st, uint64_t nlocal, uint64_t nghost, const AtomCols& c,
                    const uint32_t* ghost_root, const uint32_t* ghost_chain, const SwapConst& sc,
                    const int* fwd_planes, int nfwd, bool zero_force) {
    if (nghost == 0) return;
    PlaneList pl;
    pl.n = nfwd;
    for (int k = 0; k < nfwd; ++k) pl.idx[k] = fwd_planes[k];
    note_launch();
    k_forward<<<grid_for(nghost), kBlock, 0, st>>>(nlocal, nghost, c, ghost_root, ghost_chain, sc,
                                                   pl, zero_force ? 1 : 0);
}

__global__ void __launch_bounds__(kBlock) k_reverse_swap(uint64_t count, uint64_t recv_start,
                                                         const uint32_t* send, AtomCols c,
                                                         PlaneList rev) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t o = send[k];
        const uint64_t g = recv_start + k;
        c.fx[o] = c.fx[o] + c.fx[g];
        c.fy[o] = c.fy[o] + c.fy[g];
        c.fz[o] = c.fz[o] + c.fz[g];
        for (int q = 0; q < rev.n; ++q) c.planes[rev.idx[q]][o] = c.planes[rev.idx[q]][o] + c.planes[rev.idx[q]][g];
    }
}

void launch_reverse_swap(cudaStream_t st, uint64_t count, uint64_t recv_start,
                         const uint32_t* send, const AtomCols& c, const int* rev_planes,
                         int nrev) {
    if (count == 0) return;
    PlaneList pl;
    pl.n = nrev;
    for (int k = 0; k < nrev; ++k) pl.idx[k] = rev_planes[k];
    note_launch();
    k_reverse_swap<<<grid_for(count), kBlock, 0, st>>>(count, recv_start, send, c, pl);
}

}  // namespace soil
