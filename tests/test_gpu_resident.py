"""Device-resident communicate-only steps (k_steps): consecutive steps that
keep their lists run in one cooperative launch that stops itself when a
displacement check trips (decide_rebuild, crates/soil_core/src/neighbor.rs:
796-822).  The same workloads stepped with SOIL_RESIDENT_STEPS=1 (resident
steps at any size) and =0 (one launch per phase, a host read per step) must
be bit-identical to each other and to the CPU oracle, and the resident run
must issue far fewer kernel launches."""
import os

import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu


def _run(ctx, w, mode, chunks):
    old = os.environ.get("SOIL_RESIDENT_STEPS")
    os.environ["SOIL_RESIDENT_STEPS"] = mode
    try:
        lib = abi.load_library()
        g = system.from_workload(ctx, w)
        l0 = lib.soil_kernel_launches()
        for n in chunks:
            g.step(n)
        return g, lib.soil_kernel_launches() - l0
    finally:
        if old is None:
            del os.environ["SOIL_RESIDENT_STEPS"]
        else:
            os.environ["SOIL_RESIDENT_STEPS"] = old


CASES = {
    "plain-no-consumer": lambda: W.mono("res-plain", 81, 4096, 0.30, 1e-3, 0),
    "poly-harmonic": lambda: W.poly("res-poly", 82, 5000, 0.50, 1e-4, 0, harmonic_k=1e3),
    "poly-newton-off": lambda: W.poly("res-nn", 83, 3000, 0.45, 1e-4, 0, harmonic_k=1e3,
                                      newton=0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_resident_steps_bit_identical(ctx, name):
    w = CASES[name]()
    w.vel *= 3.0  # several rebuilds inside the run
    chunks = [1, 37, 2, 60]  # calls that end on light and rebuild steps alike
    g_res, n_res = _run(ctx, w, "1", chunks)
    g_ph, n_ph = _run(ctx, w, "0", chunks)
    o = oracle.from_workload(w)
    o.step(sum(chunks))
    for g in (g_res, g_ph):
        assert_same_state(g, o, name)
        assert_same_lists(g, o, name)
    c = g_res.counts()
    assert 3 <= c.rebuilds < sum(chunks)  # light steps ran between rebuilds
    assert n_res < n_ph, (n_res, n_ph)
    g_res.close()
    g_ph.close()


def test_resident_light_steps_take_one_launch(ctx):
    """Without rebuilds, a call of 40 steps is one resident launch (plus the
    final half-kick), against two or more launches per step phase by phase."""
    w = W.poly("res-light", 85, 4000, 0.45, 1e-5, 0, harmonic_k=1e3)
    g_res, n_res = _run(ctx, w, "1", [1, 40])
    g_ph, n_ph = _run(ctx, w, "0", [1, 40])
    assert g_res.counts().rebuilds == 1  # the setup build only
    assert_same_state(g_res, g_ph)
    l_res, l_ph = _launches_of(ctx, g_res, 40), _launches_of(ctx, g_ph, 40, mode="0")
    assert l_res <= 4 and l_ph >= 80, (l_res, l_ph)
    g_res.close()
    g_ph.close()


def _launches_of(ctx, g, n, mode="1"):
    old = os.environ.get("SOIL_RESIDENT_STEPS")
    os.environ["SOIL_RESIDENT_STEPS"] = mode
    try:
        lib = abi.load_library()
        l0 = lib.soil_kernel_launches()
        g.step(n)
        return lib.soil_kernel_launches() - l0
    finally:
        if old is None:
            del os.environ["SOIL_RESIDENT_STEPS"]
        else:
            os.environ["SOIL_RESIDENT_STEPS"] = old


def test_resident_steps_stop_at_the_periodic_sort(ctx):
    """A periodic sort falls due on a light step: the resident launch must
    end before it so the host runs the sort."""
    w = W.poly("res-sort", 84, 3000, 0.45, 1e-4, 0, harmonic_k=1e3, sort_every=7)
    g, _ = _run(ctx, w, "1", [40])
    o = oracle.from_workload(w)
    o.step(40)
    assert_same_state(g, o)
    assert_same_lists(g, o)
    np.testing.assert_array_equal(g.sort_perm(), o.sort_perm())
    g.close()
