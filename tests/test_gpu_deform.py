"""Orthogonal box deformation (soil_sys_set_deform; apply_deform,
soil_deform/src/lib.rs:468-557) against the CPU oracle, bit for bit: erate
compression, vel expansion and a final-style ramp, with and without the
position remap, alone and combined with Lees-Edwards shear.  The oracle's
deform is pinned to the reference's own tests (test_oracle_known_answers)."""
import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu

CASES = {
    # name: ([(dim, style, a, b, stage)], remap, shear)
    "erate-z-compress": ([(2, abi.SOIL_DEFORM_ERATE, -2.0, 0.0, 0)], True, 0.0),
    "vel-x-expand": ([(0, abi.SOIL_DEFORM_VEL, 3.0, 0.0, 0)], True, 0.0),
    "final-y-ramp": ([(1, abi.SOIL_DEFORM_FINAL, 0.4, None, 30)], True, 0.0),
    "erate-xz-no-remap": ([(0, abi.SOIL_DEFORM_ERATE, 0.5, 0.0, 0),
                           (2, abi.SOIL_DEFORM_ERATE, -0.5, 0.0, 0)], False, 0.0),
    "erate-z-with-shear": ([(2, abi.SOIL_DEFORM_ERATE, -1.0, 0.0, 0)], True, 1.5),
}


def _pair(ctx, w, axes, remap):
    g = system.System(ctx, w.box, w.cfg, w.dt)
    o = oracle.OracleSystem(w.box, w.cfg, w.dt)
    for s in (g, o):
        rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
        s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
        s.set_harmonic(w.harmonic_k, rc)
        if w.shear_rate:
            s.set_shear(w.shear_rate)
        for dim, style, a, b, stage in axes:
            if b is None:  # final: target [lo + a, hi - a]
                lo, hi = w.box.lo[dim], w.box.hi[dim]
                a, b = lo + a, hi - a
            s.set_deform(dim, style, a, b, stage)
        s.set_deform_remap(remap)
        s.setup()
    return g, o


@pytest.mark.parametrize("name", list(CASES))
def test_deform_matches_oracle(ctx, name):
    axes, remap, shear = CASES[name]
    w = W.poly("deform", 31, 3000, 0.45, 1e-3, 40, harmonic_k=1e3, shear_rate=shear)
    g, o = _pair(ctx, w, axes, remap)
    g.step(17)
    o.step(17)
    g.step(23)
    o.step(23)
    assert_same_state(g, o, name)
    assert_same_lists(g, o, name)
    lg, hg, tg = g.box()
    lo, ho, to = o.box()
    for a, b in ((lg, lo), (hg, ho), (tg, to)):
        np.testing.assert_array_equal(a.view(np.uint64), b.view(np.uint64), err_msg=name)
    # the box really moved, and every deforming step rebuilt the lists
    assert np.any(lg != np.array([w.box.lo[d] for d in range(3)]))
    assert g.counts().rebuilds >= 40
    g.close()


def test_deform_collapse_fails_the_step(ctx):
    w = W.poly("collapse", 32, 500, 0.3, 0.05, 10, harmonic_k=1e3)
    g = system.System(ctx, w.box, w.cfg, w.dt)
    rc = g.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    g.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    g.set_harmonic(w.harmonic_k, rc)
    g.set_deform(0, abi.SOIL_DEFORM_ERATE, -25.0)  # 1 - 1.25 step: negative at step 1
    g.setup()
    with pytest.raises(abi.SoilError, match="collapsed"):
        g.step(1)
    g.close()


def test_deform_is_refused_after_setup_and_in_a_batch(ctx):
    w = W.config4_box(2, nmin=256, nmax=600, steps=5)
    s = system.from_workload(ctx, w)
    with pytest.raises(abi.SoilError):
        s.set_deform(0, abi.SOIL_DEFORM_ERATE, 0.1)
    s.close()
    g = system.System(ctx, w.box, w.cfg, w.dt)
    rc = g.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    g.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    g.set_harmonic(w.harmonic_k, rc)
    g.set_deform(1, abi.SOIL_DEFORM_VEL, 0.5)
    g.setup()
    b = system.Batch(ctx)
    with pytest.raises(abi.SoilError):
        b.add(g)
    b.close()
    g.close()
