// k_neighbor.cu — half-list CSR build of bin_neighbor_list
// (neighbor.rs:1127-1319) and the transposed ("incoming") lists the
// deterministic force gather reads.
//
// Row order is the reference's: the self-cell tail (sorted slots after the
// atom's own slot), then every forward-stencil cell in stencil order, each
// cell in sorted (ascending index) order.  A count pass sizes the rows, an
// exclusive scan gives neighbor_offsets, a fill pass writes the indices.
//
// Filter: FP64 `fma(dx,dx,fma(dy,dy,dz*dz)) < cut^2` exactly as the
// reference, or (FP32 mode) a float test on grid-relative coordinates that
// only REJECTS candidates provably outside the cutoff — the margin eps bounds
// the float rounding of coordinates, differences and squares — followed by
// the exact FP64 test on the rest, so the lists are identical in both modes.
#include "kernels.cuh"

namespace soil {

template <bool UNIFORM, bool FP32, bool FILL>
__global__ void __launch_bounds__(kBlock) k_pairs(uint64_t nlocal, AtomCols c, PairParams p,
                                                  uint32_t* rowcount, const uint32_t* offsets,
                                                  uint32_t* indices, DevFlags* flags) {
    uint64_t n_cand = 0, n_rechk = 0;
    float lim_uniform = 0.0f;
    if (UNIFORM && FP32) {
        const float cut = (float)sqrt(p.cut_sq) + p.eps32;
        lim_uniform = cut * cut;
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlocal;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t my_cell = p.atom_cell[i];
        const double pix = c.x[i], piy = c.y[i], piz = c.z[i];
        const double si = c.cut[i];
        float pix32 = 0.f, piy32 = 0.f, piz32 = 0.f, si32 = 0.f;
        if (FP32) {
            pix32 = (float)(pix - p.origin[0]);
            piy32 = (float)(piy - p.origin[1]);
            piz32 = (float)(piz - p.origin[2]);
            si32 = (float)si;
        }
        uint32_t cnt = 0;
        uint32_t out = FILL ? offsets[i] : 0u;

        auto test = [&](uint32_t m) -> bool {
            if (FP32) {
                if (!FILL) ++n_cand;
                const float dx = p.spx32[m] - pix32;
                const float dy = p.spy32[m] - piy32;
                const float dz = p.spz32[m] - piz32;
                const float r2 = dx * dx + dy * dy + dz * dz;
                float lim = lim_uniform;
                if (!UNIFORM) {
                    const float cu = (si32 + p.scut32[m]) * (float)p.sf + p.eps32;
                    lim = cu * cu;
                }
                if (r2 > lim) return false;
                if (!FILL) ++n_rechk;
            } else if (!FILL) {
                ++n_cand;
            }
            const double dx = p.spx[m] - pix;
            const double dy = p.spy[m] - piy;
            const double dz = p.spz[m] - piz;
            const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
            if (UNIFORM) return r2 < p.cut_sq;
            const double sum_skin = si + p.scut[m];
            return r2 < sum_skin * sum_skin * p.sf_sq;
        };
        auto take = [&](uint32_t m) {
            if (FILL) indices[out++] = p.sorted_atoms[m];
            else ++cnt;
        };

        if (p.has_self) {
            const uint32_t e = p.bin_start[my_cell + 1];
            if (p.newton) {
                for (uint32_t m = p.atom_sorted_idx[i] + 1; m < e; ++m)
                    if (test(m)) take(m);
            } else {
                for (uint32_t m = p.bin_start[my_cell]; m < e; ++m) {
                    if (p.sorted_atoms[m] == (uint32_t)i) continue;
                    if (test(m)) take(m);
                }
            }
        }
        for (int s = 0; s < p.nstencil; ++s) {
            const int32_t off = p.stencil[s];
            if (!p.newton && off == 0) continue;
            const uint32_t cc = (uint32_t)((int32_t)my_cell + off);
            if (cc >= p.ncells) {  // the grid's ghost layers make this unreachable
                if (flags) atomicOr(&flags->error, 1u);
                continue;
            }
            const uint32_t b = p.bin_start[cc], e = p.bin_start[cc + 1];
            for (uint32_t m = b; m < e; ++m)
                if (test(m)) take(m);
        }
        if (!FILL) rowcount[i] = cnt;
    }
    if (!FILL) {
        for (int o = 16; o > 0; o >>= 1) {
            n_cand += __shfl_down_sync(0xffffffffu, n_cand, o);
            n_rechk += __shfl_down_sync(0xffffffffu, n_rechk, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd((unsigned long long*)&flags->candidates, (unsigned long long)n_cand);
            atomicAdd((unsigned long long*)&flags->rechecked, (unsigned long long)n_rechk);
        }
    }
}

template <bool FILL>
static void dispatch_pairs(cudaStream_t st, uint64_t nlocal, const AtomCols& c, const PairParams& p,
                           uint32_t* rowcount, const uint32_t* offsets, uint32_t* indices,
                           DevFlags* flags) {
    const unsigned g = grid_for(nlocal);
    const bool fp32 = p.filter == SOIL_FILTER_FP32_RECHECK;
    note_launch();
    if (p.uniform) {
        if (fp32) k_pairs<true, true, FILL><<<g, kBlock, 0, st>>>(nlocal, c, p, rowcount, offsets, indices, flags);
        else k_pairs<true, false, FILL><<<g, kBlock, 0, st>>>(nlocal, c, p, rowcount, offsets, indices, flags);
    } else {
        if (fp32) k_pairs<false, true, FILL><<<g, kBlock, 0, st>>>(nlocal, c, p, rowcount, offsets, indices, flags);
        else k_pairs<false, false, FILL><<<g, kBlock, 0, st>>>(nlocal, c, p, rowcount, offsets, indices, flags);
    }
}

void launch_pair_count(cudaStream_t st, uint64_t nlocal, const AtomCols& c, const PairParams& p,
                       uint32_t* rowcount, DevFlags* flags) {
    if (nlocal == 0) return;
    dispatch_pairs<false>(st, nlocal, c, p, rowcount, nullptr, nullptr, flags);
}

void launch_pair_fill(cudaStream_t st, uint64_t nlocal, const AtomCols& c, const PairParams& p,
                      const uint32_t* offsets, uint32_t* indices) {
    if (nlocal == 0) return;
    dispatch_pairs<true>(st, nlocal, c, p, nullptr, offsets, indices, nullptr);
}

__global__ void __launch_bounds__(kBlock) k_in_count(uint64_t nlocal, const uint32_t* offsets,
                                                     const uint32_t* indices, uint32_t* incount) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlocal;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (uint32_t q = offsets[i]; q < offsets[i + 1]; ++q) atomicAdd(&incount[indices[q]], 1u);
}

void launch_in_count(cudaStream_t st, uint64_t nlocal, const uint32_t* offsets,
                     const uint32_t* indices, uint32_t* incount) {
    if (nlocal == 0) return;
    note_launch();
    k_in_count<<<grid_for(nlocal), kBlock, 0, st>>>(nlocal, offsets, indices, incount);
}

__global__ void __launch_bounds__(kBlock) k_in_scatter(uint64_t nlocal, const uint32_t* offsets,
                                                       const uint32_t* indices, uint32_t* cursor,
                                                       uint32_t* in_list) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nlocal;
         i += (uint64_t)gridDim.x * blockDim.x)
        for (uint32_t q = offsets[i]; q < offsets[i + 1]; ++q)
            in_list[atomicAdd(&cursor[indices[q]], 1u)] = (uint32_t)i;
}

void launch_in_scatter(cudaStream_t st, uint64_t nlocal, const uint32_t* offsets,
                       const uint32_t* indices, uint32_t* cursor, uint32_t* in_list) {
    if (nlocal == 0) return;
    note_launch();
    k_in_scatter<<<grid_for(nlocal), kBlock, 0, st>>>(nlocal, offsets, indices, cursor, in_list);
}

}  // namespace soil
