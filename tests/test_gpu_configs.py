"""Bit-exact parity with the CPU oracle at the benchmark configurations' full
sizes, through their natural neighbor rebuilds:

  32,768-atom plain box (phi 0.30, F = 0, dt 1e-3): all 2,000 steps, compared
      at steps 1,000 and 2,000 (~180 rebuilds);
  4,194,304-atom polydisperse box (phi 0.50, harmonic k = 1e3, dt 1e-4): every
      step up to five steps past the first rebuild after the setup build (the
      first falls near step 50), in the FP64 and FP32+FP64-recheck filters;
  1,048,576-atom Lees-Edwards box (phi 0.40, xy rate 0.1, k = 1e3, dt 1e-4):
      20 sheared steps, each a full rebuild of the tilted grid.

Compared as IEEE bit patterns: positions, velocities, forces, images, tags,
ghost origins, the radius column, CSR offsets and indices (order included),
swap send lists, recv ranges and offsets, and the spatial-sort permutation.
The stated trajectory tolerance is 1e-12 relative; these tests demand 0."""
import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu


def _compare(g, o, what):
    assert_same_state(g, o, what)
    assert_same_lists(g, o, what)
    np.testing.assert_array_equal(g.sort_perm(), o.sort_perm(), err_msg=f"{what} sort_perm")


def test_plain_32768_all_2000_steps(ctx):
    w = W.config1()
    assert (w.n, w.steps) == (32768, 2000)
    g, o = system.from_workload(ctx, w), oracle.from_workload(w)
    for k in range(2):
        g.step(1000)
        o.step(1000)
        _compare(g, o, f"plain after {1000 * (k + 1)} steps")
    assert g.counts().rebuilds > 100
    g.close()


@pytest.mark.parametrize("filt", [abi.SOIL_FILTER_FP64, abi.SOIL_FILTER_FP32_RECHECK])
def test_large_4194304_through_a_natural_rebuild(ctx, filt):
    w = W.config2(filt=filt)
    assert w.n == 4194304
    o = oracle.from_workload(w)
    steps = 0
    while o.counts().rebuilds < 2 and steps < 200:  # the setup build, then a natural one
        o.step(1)
        steps += 1
    assert o.counts().rebuilds == 2, "no natural rebuild within 200 steps"
    o.step(5)
    steps += 5
    g = system.from_workload(ctx, w)
    g.step(steps)
    _compare(g, o, f"large box after {steps} steps")
    c = g.counts()
    if filt == abi.SOIL_FILTER_FP32_RECHECK:
        assert 0 < c.filter_rechecked < c.filter_candidates
    g.close()


def test_shear_1048576_twenty_steps(ctx):
    w = W.config3()
    assert w.n == 1048576 and w.shear_rate == 0.1
    g, o = system.from_workload(ctx, w), oracle.from_workload(w)
    for k in range(2):
        g.step(10)
        o.step(10)
        _compare(g, o, f"sheared box after {10 * (k + 1)} steps")
    c = g.counts()
    assert c.triclinic and c.tilt_xy != 0.0 and c.rebuilds == 20
    g.close()
