"""Bit-exact parity of the CUDA path with the CPU oracle on seeded inputs.

Every observable the reference exposes is compared after N steps: atom
state (pos/vel/force/image/tag/origin as IEEE bit patterns), the CSR
neighbor list (offsets and indices, order included), the ghost swap maps,
the spatial-sort permutation and the counters.  Trajectory tolerance stated
for this path is 1e-12 relative; these tests demand 0.
"""
import numpy as np
import pytest

from helpers import assert_same_lists, assert_same_state, pair
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu


def test_config1_plain_small(ctx):
    w = W.config1(n=4096, steps=60)
    g, o = pair(ctx, w)
    for k in range(3):
        g.step(20)
        o.step(20)
        assert_same_state(g, o, f"after {20 * (k + 1)} steps")
        assert_same_lists(g, o)
    np.testing.assert_array_equal(g.sort_perm(), o.sort_perm())
    assert g.counts().rebuilds > 2


def test_poly_harmonic_fp64(ctx):
    w = W.poly("poly", 7, 6000, 0.5, 1e-4, 100, harmonic_k=1e3)
    g, o = pair(ctx, w)
    g.step(100)
    o.step(100)
    assert_same_state(g, o)
    assert_same_lists(g, o)
    assert np.any(g.atoms()["force"] != 0.0)


def test_poly_harmonic_fp32_recheck_equals_fp64(ctx):
    w = W.poly("poly32", 8, 6000, 0.5, 1e-4, 60, harmonic_k=1e3,
               filter=abi.SOIL_FILTER_FP32_RECHECK)
    g, o = pair(ctx, w)
    g.step(60)
    o.step(60)
    assert_same_state(g, o)
    assert_same_lists(g, o)
    c = g.counts()
    assert c.filter_candidates > 0 and 0 < c.filter_rechecked < c.filter_candidates


def test_shear_lees_edwards(ctx):
    # fast shear so the tilt wraps (box flip) inside the run
    w = W.mono("shear", 9, 4000, 0.4, 1e-3, 120, harmonic_k=1e3, shear_rate=5.0)
    g, o = pair(ctx, w)
    for k in range(4):
        g.step(30)
        o.step(30)
        assert_same_state(g, o, f"shear step {30 * (k + 1)}")
        assert_same_lists(g, o)
    assert g.counts().triclinic == 1


def test_periodic_sort_and_every_check(ctx):
    w = W.mono("sort", 10, 3000, 0.3, 1e-3, 50, sort_every=7, every=5, check=1)
    g, o = pair(ctx, w)
    for k in range(5):
        g.step(10)
        o.step(10)
        assert_same_state(g, o, f"step {10 * (k + 1)}")
        assert_same_lists(g, o)


def test_every_without_check(ctx):
    w = W.mono("every", 11, 2000, 0.3, 1e-3, 30, every=4, check=0)
    g, o = pair(ctx, w)
    g.step(30)
    o.step(30)
    assert_same_state(g, o)
    assert_same_lists(g, o)


def test_newton_off_full_list(ctx):
    w = W.poly("full", 12, 3000, 0.45, 1e-4, 40, harmonic_k=1e3, newton=0)
    g, o = pair(ctx, w)
    g.step(40)
    o.step(40)
    assert_same_state(g, o)
    assert_same_lists(g, o)


def test_small_box_multiple_images(ctx):
    # box barely larger than the ghost cutoff: atoms near both faces, corner
    # ghosts of ghosts (chains of length 3), self-images in the list
    w = W.mono("tiny", 13, 40, 0.3, 1e-3, 25, harmonic_k=1e3)
    g, o = pair(ctx, w)
    g.step(25)
    o.step(25)
    assert_same_state(g, o)
    assert_same_lists(g, o)


def test_phase_by_phase(ctx):
    w = W.poly("phases", 14, 2500, 0.5, 1e-4, 0, harmonic_k=1e3, shear_rate=0.5)
    g, o = pair(ctx, w)
    for step in range(6):
        for ph in abi.PHASES:
            g.phase(ph)
            o.phase(ph)
            assert_same_state(g, o, f"step {step} after {ph}")
    assert_same_lists(g, o)


def test_single_atom_and_empty_rows(ctx):
    w = W.mono("one", 15, 1, 0.01, 1e-3, 10)
    g, o = pair(ctx, w)
    g.step(10)
    o.step(10)
    assert_same_state(g, o)
    assert_same_lists(g, o)


def test_empty_system_steps_like_the_oracle(ctx):
    """No atoms at all: setup, steps (each a rebuild, as the reference's
    needs_rebuild says for nlocal == 0) and readbacks work and match."""
    import oracle as orc
    b = W.make_box(10.0)
    g = system.System(ctx, b, W.default_cfg(), 1e-3)
    o = orc.OracleSystem(b, W.default_cfg(), 1e-3)
    for s in (g, o):
        rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
        s.add_atoms(np.zeros(0, np.uint32), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0),
                    np.zeros(0), columns=[np.zeros(0)])
        s.set_harmonic(1e3, rc)
        s.setup()
        s.step(2)
        s.step(3)
    assert_same_state(g, o, "empty")
    assert_same_lists(g, o, "empty")
    assert g.counts().nlocal == 0 and g.counts().step == 5
    g.close()
