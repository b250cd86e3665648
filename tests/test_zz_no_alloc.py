"""soil_bin_sort_noalloc against the spatial sort of soil_phase_sort.

soil_bin_sort_noalloc exists for hosts that cannot allocate device memory
while they run (a fixed HBM plan, or an allocator that owns the device): it
takes caller-owned device buffers and keeps its own scratch in a static
device array.  This test calls it through the C ABI on the positions a
system holds right before its sort phase and checks that its permutation
equals the one soil_phase_sort applies (integer output: exact equality).
It does so for two systems in a row, the second with a smaller bin grid,
so a histogram left over from the first call would show up as a mismatch,
and once more on a sheared (triclinic) box a few steps in, where cells are
computed in lamda coordinates from the box's current tilt.
The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu


def _dptr(t):
    return C.c_void_p(t.data_ptr())


def _arr(vals, ct):
    return (ct * 3)(*vals)


def _sort_both_ways(ctx, w):
    g = system.from_workload(ctx, w)
    o = oracle.from_workload(w)  # same grid as the GPU system; used for origin / bin size
    _, origin, bin_size = o.stencil()
    counts = g.counts()
    assert list(counts.bin_count) == list(o.counts().bin_count)
    # run the first step up to (not including) its sort phase
    for ph in ("deform", "initial", "decide_rebuild", "remove_ghosts", "zero_forces", "pbc"):
        g.phase(ph)
    a = g.atoms(local_only=True)
    n = len(a["tag"])
    dev = torch.device("cuda", 0)
    x = torch.tensor(a["pos"][:, 0].copy(), dtype=torch.float64, device=dev)
    y = torch.tensor(a["pos"][:, 1].copy(), dtype=torch.float64, device=dev)
    z = torch.tensor(a["pos"][:, 2].copy(), dtype=torch.float64, device=dev)
    cell = torch.full((n,), -1, dtype=torch.int32, device=dev)
    perm = torch.full((n,), -1, dtype=torch.int32, device=dev)
    box_lo = [w.box.lo[d] for d in range(3)]
    box_size = [w.box.hi[d] - w.box.lo[d] for d in range(3)]
    torch.cuda.synchronize()
    st = ctx.lib.soil_bin_sort_noalloc(
        ctx.h, _dptr(x), _dptr(y), _dptr(z), n,
        _arr(origin, C.c_double), _arr(bin_size, C.c_double),
        _arr(list(counts.bin_count), C.c_int32),
        _arr(box_lo, C.c_double), _arr(box_size, C.c_double), _arr([0.0, 0.0, 0.0], C.c_double),
        0, _dptr(cell), _dptr(perm), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.SOIL_OK, ctx.error()
    torch.cuda.synchronize()
    got = perm.cpu().numpy().view(np.uint32)
    got_cell = cell.cpu().numpy().view(np.uint32)
    g.phase("sort")  # the existing entry point
    want = g.sort_perm()
    g.close()
    return got, got_cell, want


def test_no_alloc_sort_matches_phase_sort_twice(ctx):
    first = W.poly("noalloc-a", 31, 30000, 0.45, 1e-4, 0)    # larger grid
    second = W.mono("noalloc-b", 32, 5000, 0.30, 1e-3, 0)    # smaller grid, reuses the scratch
    for w in (first, second):
        got, got_cell, want = _sort_both_ways(ctx, w)
        np.testing.assert_array_equal(got, want)
        # cells come back in original atom order and are sorted by the permutation
        assert np.all(np.diff(got_cell[got].astype(np.int64)) >= 0)


def test_no_alloc_sort_matches_phase_sort_sheared(ctx):
    """Lamda binning: the box is tilted by the shear drive; the grid is the
    one the oracle's sort uses on the same step (recomputed from the tilt)."""
    w = W.mono("noalloc-shear", 33, 6000, 0.40, 1e-3, 0, harmonic_k=1e3, shear_rate=0.5)
    g = system.from_workload(ctx, w)
    o = oracle.from_workload(w)
    g.step(3)
    o.step(3)
    pre = ("deform", "initial", "decide_rebuild", "remove_ghosts", "zero_forces", "pbc")
    for ph in pre:
        g.phase(ph)
        o.phase(ph)
    o.phase("sort")  # recomputes the bin grid from the tilt, as the GPU sort will
    _, origin, bin_size = o.stencil()
    bin_count = list(o.counts().bin_count)
    lo, hi, tilt = g.box()
    assert tilt[0] != 0.0
    a = g.atoms(local_only=True)
    n = len(a["tag"])
    dev = torch.device("cuda", 0)
    x, y, z = (torch.tensor(a["pos"][:, d].copy(), dtype=torch.float64, device=dev)
               for d in range(3))
    cell = torch.full((n,), -1, dtype=torch.int32, device=dev)
    perm = torch.full((n,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    st = ctx.lib.soil_bin_sort_noalloc(
        ctx.h, _dptr(x), _dptr(y), _dptr(z), n, _arr(origin, C.c_double),
        _arr(bin_size, C.c_double), _arr(bin_count, C.c_int32), _arr(lo, C.c_double),
        _arr(hi - lo, C.c_double), _arr(tilt, C.c_double), 1, _dptr(cell), _dptr(perm),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.SOIL_OK, ctx.error()
    torch.cuda.synchronize()
    got = perm.cpu().numpy().view(np.uint32)
    g.phase("sort")
    assert list(g.counts().bin_count) == bin_count
    np.testing.assert_array_equal(got, g.sort_perm())
    np.testing.assert_array_equal(got, o.sort_perm())
    g.close()


def test_no_alloc_sort_rejects_oversized_grid(ctx):
    one = (C.c_double * 3)(1.0, 1.0, 1.0)
    zero = (C.c_double * 3)(0.0, 0.0, 0.0)
    big = (C.c_int32 * 3)(200, 200, 200)  # 8,000,000 cells > 2,097,152
    st = ctx.lib.soil_bin_sort_noalloc(ctx.h, None, None, None, 0, zero, one, big, zero, one,
                                       zero, 0, None, None, None)
    assert st == abi.SOIL_ERR_CAPACITY
    assert "exceed the fixed scratch limit" in ctx.error()
