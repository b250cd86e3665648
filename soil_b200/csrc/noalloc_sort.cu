// noalloc_sort.cu — the spatial sort's stable counting sort by bin cell,
// for callers that cannot allocate device memory.
//
// Some hosts fix all device memory up front: a serving loop that admits
// systems against a planned HBM budget, or an embedding application whose
// allocator owns the whole device and forbids allocation once stepping has
// started (a cudaMalloc/cudaFree there would also synchronise the device and
// stall every other stream).  soil_bin_sort_noalloc gives them the same
// permutation as the spatial sort of soil_phase_sort without allocating:
// the caller passes positions, the per-atom cell output and the permutation
// output; the cell histogram, its scan and the scan's tile sums live in one
// file-scope device array of fixed size (kNoAllocScratchWords u32, 16 MiB),
// which every GPU that loads this library keeps until the process exits.
//
// The scratch is shared by every call on a device and keeps the previous
// call's contents; each call clears the histogram it uses before counting.
// Calls whose work overlaps on the GPU (two streams, or two host threads)
// race on that array and must be serialised by the caller.
#include <cstdio>
#include <cstring>

#include "kernels.cuh"

struct soil_ctx;  // defined in soil_capi.cu

namespace soil {
int set_ctx_error(soil_ctx* ctx, int status, const char* msg);
}

namespace {

using namespace soil;

// Largest bin grid served: 2^21 = 2,097,152 cells.  The 32,768-atom box
// (41^3 cells), the 1,048,576-atom sheared box (~107^3) and every batched or
// served box fit; the 4,194,304-atom box at its default grid (133^3 cells)
// does not and gets SOIL_ERR_CAPACITY.
constexpr uint64_t kNoAllocMaxCells = 1ull << 21;
// histogram/cursor (cells+1) + scan output (cells+2) + scan tile sums
constexpr uint64_t kNoAllocScratchWords =
    (kNoAllocMaxCells + 1) + (kNoAllocMaxCells + 2) + (kNoAllocMaxCells / 2048 + 2);

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocScratchWords];

// Device address of g_noalloc_scratch on the current device.  The host-side
// name of the array is only a stand-in for the symbol, not a device address.
// The address is looked up on every call (the lookup is cheap), so a module
// reloaded after cudaDeviceReset is never reached through a stale pointer.
int scratch_for_current_device(soil_ctx* ctx, uint32_t** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return set_ctx_error(ctx, SOIL_ERR_NO_DEVICE, "soil_bin_sort_noalloc: no current CUDA device");
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        char buf[160];
        snprintf(buf, sizeof buf, "soil_bin_sort_noalloc: cudaGetSymbolAddress failed: %s",
                 cudaGetErrorString(e));
        return set_ctx_error(ctx, SOIL_ERR_CUDA, buf);
    }
    *out = (uint32_t*)p;
    return SOIL_OK;
}

}  // namespace

extern "C" int soil_bin_sort_noalloc(soil_ctx* ctx, const double* d_x, const double* d_y,
                                     const double* d_z, uint64_t n, const double origin[3],
                                     const double bin_size[3], const int32_t bin_count[3],
                                     const double box_lo[3], const double box_size[3],
                                     const double tilt[3], int32_t triclinic, uint32_t* d_cell,
                                     uint32_t* d_perm, void* stream) {
    if (!origin || !bin_size || !bin_count || !box_lo || !box_size || !tilt)
        return set_ctx_error(ctx, SOIL_ERR_INVALID, "soil_bin_sort_noalloc: null grid argument");
    if (n && (!d_x || !d_y || !d_z || !d_cell || !d_perm))
        return set_ctx_error(ctx, SOIL_ERR_INVALID, "soil_bin_sort_noalloc: null device pointer");
    for (int d = 0; d < 3; ++d)
        if (bin_count[d] < 1 || !(bin_size[d] > 0.0) || !(box_size[d] > 0.0))
            return set_ctx_error(ctx, SOIL_ERR_INVALID, "soil_bin_sort_noalloc: invalid bin grid");
    // the product is built factor by factor and stops past the limit, so
    // counts whose 64-bit product would wrap are refused too
    uint64_t ncells = 1;
    for (int d = 0; d < 3 && ncells <= kNoAllocMaxCells; ++d) ncells *= (uint64_t)bin_count[d];
    if (ncells > kNoAllocMaxCells) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "soil_bin_sort_noalloc: %llu bin cells exceed the fixed scratch limit of %llu "
                 "cells; use soil_phase_sort (which allocates) for this grid",
                 (unsigned long long)ncells, (unsigned long long)kNoAllocMaxCells);
        return set_ctx_error(ctx, SOIL_ERR_CAPACITY, buf);
    }
    if (n >= 0x7fffffffull)
        return set_ctx_error(ctx, SOIL_ERR_CAPACITY, "soil_bin_sort_noalloc: n exceeds the u32 index range");
    uint32_t* scratch = nullptr;
    int r = scratch_for_current_device(ctx, &scratch);
    if (r != SOIL_OK) return r;
    if (n == 0) return SOIL_OK;

    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* counts = scratch;                      // histogram, then cursor
    uint32_t* start = scratch + (kNoAllocMaxCells + 1);
    uint32_t* partials = start + (kNoAllocMaxCells + 2);

    Grid gr;
    for (int d = 0; d < 3; ++d) {
        gr.origin[d] = origin[d];
        gr.inv_bs[d] = 1.0 / bin_size[d];
        gr.n[d] = bin_count[d];
        gr.geom.lo[d] = box_lo[d];
        gr.geom.size[d] = box_size[d];
        gr.geom.tilt[d] = tilt[d];
    }
    gr.geom.triclinic = triclinic ? 1 : 0;
    AtomCols c;
    std::memset(&c, 0, sizeof c);
    c.x = const_cast<double*>(d_x);
    c.y = const_cast<double*>(d_y);
    c.z = const_cast<double*>(d_z);

    cudaError_t e = cudaMemsetAsync(counts, 0, ncells * sizeof(uint32_t), st);
    if (e == cudaSuccess) {
        launch_cells(st, 0, n, c, gr, d_cell, counts);
        exclusive_scan_u32(st, counts, start, ncells, partials);
        e = cudaMemcpyAsync(counts, start, ncells * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    }
    if (e == cudaSuccess) {
        launch_scatter(st, n, d_cell, counts, d_perm);
        launch_segsort(st, ncells, start, d_perm);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        char buf[200];
        snprintf(buf, sizeof buf, "soil_bin_sort_noalloc: %s", cudaGetErrorString(e));
        return set_ctx_error(ctx, SOIL_ERR_CUDA, buf);
    }
    return SOIL_OK;
}
