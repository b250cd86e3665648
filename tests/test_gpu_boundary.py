"""Fixed and shrink-wrapped boundaries (soil_sys_set_boundary) against the CPU
oracle, bit for bit: atoms leaving a fixed axis are removed by pbc in the
reference's swap-remove order, swaps of a non-periodic axis pack their face
atoms but receive nothing, shrink-wrapped axes follow the atoms every step
(a rebuild each time they move), and the displacement check takes the
general per-axis path.  The oracle's boundary code is pinned to the
reference's own tests (test_oracle_known_answers)."""
import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu
P, F, S = abi.SOIL_BOUNDARY_PERIODIC, abi.SOIL_BOUNDARY_FIXED, abi.SOIL_BOUNDARY_SHRINK

CASES = {
    # name: (types, padding, velocity scale, newton, shear rate)
    "fixed-z": ([P, P, F], 0.0, 25.0, 1, 0.0),
    "fixed-xyz": ([F, F, F], 0.0, 25.0, 1, 0.0),
    "shrink-z": ([P, P, S], 0.0, 3.0, 1, 0.0),
    "shrink-xy-padded": ([S, S, P], 0.7, 3.0, 1, 0.0),
    "fixed-x-shrink-z-newton-off": ([F, P, S], 0.0, 10.0, 0, 0.0),
    # Lees-Edwards shear with walls in z: triclinic wrap and lamda face tests
    "sheared-fixed-z": ([P, P, F], 0.0, 25.0, 1, 2.0),
    "sheared-shrink-z": ([P, P, S], 0.5, 3.0, 1, 2.0),
}


def _pair(ctx, w, types, padding):
    g = system.System(ctx, w.box, w.cfg, w.dt)
    o = oracle.OracleSystem(w.box, w.cfg, w.dt)
    for s in (g, o):
        rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
        s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
        s.set_harmonic(w.harmonic_k, rc)
        if w.shear_rate:
            s.set_shear(w.shear_rate)
        s.set_boundary(types, padding)
        s.setup()
    return g, o


@pytest.mark.parametrize("name", list(CASES))
def test_boundaries_match_oracle(ctx, name):
    types, padding, vscale, newton, shear = CASES[name]
    w = W.poly("bounds", 41, 3000, 0.4, 1e-3, 40, harmonic_k=1e3, shear_rate=shear)
    w.vel *= vscale
    w.cfg.newton = newton
    g, o = _pair(ctx, w, types, padding)
    for k in (13, 27):
        g.step(k)
        o.step(k)
        assert_same_state(g, o, name)
        assert_same_lists(g, o, name)
    lg, hg, _ = g.box()
    lo, ho, _ = o.box()
    np.testing.assert_array_equal(lg.view(np.uint64), lo.view(np.uint64), err_msg=name)
    np.testing.assert_array_equal(hg.view(np.uint64), ho.view(np.uint64), err_msg=name)
    sw = g.swaps()
    for d in range(3):
        if types[d] != P:  # packed but nothing received, no shift
            for k in (2 * d, 2 * d + 1):
                assert sw[k]["recv_count"] == 0 and np.all(sw[k]["offset"] == 0.0)
            assert len(sw[2 * d]["send"]) + len(sw[2 * d + 1]["send"]) > 0
    c = g.counts()
    if F in types:
        assert c.nlocal < w.n, "no atom left through a fixed face"
    if S in types or shear:
        assert c.rebuilds >= 40  # the bounds or the tilt move every step
    g.close()


def test_boundary_refusals(ctx):
    w = W.poly("bounds-bad", 42, 500, 0.3, 1e-3, 5, harmonic_k=1e3, shear_rate=1.0)
    g = system.System(ctx, w.box, w.cfg, w.dt)
    rc = g.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    g.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    g.set_harmonic(w.harmonic_k, rc)
    with pytest.raises(abi.SoilError):
        g.set_boundary([P, P, 3])
    g.set_shear(1.0)
    g.set_boundary([P, F, P])
    with pytest.raises(abi.SoilError, match="periodic"):
        g.setup()  # Lees-Edwards shear needs periodic x and y
    g.close()
    s = system.from_workload(ctx, W.config4_box(3, nmin=256, nmax=600, steps=5))
    with pytest.raises(abi.SoilError):
        s.set_boundary([P, P, F])  # after setup
    s.close()


def test_every_atom_leaves_a_fixed_box(ctx):
    """Atoms fast enough to leave a fully fixed box within a few steps: the
    system empties exactly as the oracle's, and keeps stepping with no atoms."""
    w = W.mono("escape", 43, 200, 0.2, 1e-2, 30)
    w.vel *= 200.0
    g, o = _pair(ctx, w, [F, F, F], 0.0)
    for k in (3, 7, 20):
        g.step(k)
        o.step(k)
        assert_same_state(g, o, f"escape +{k}")
    assert g.counts().nlocal == 0 and g.counts().nghost == 0
    g.close()
