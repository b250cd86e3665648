"""The rebuild path's speed switches change no result: the pair scan with
range bounds loaded as it goes (SOIL_PAIRS_PRE=0), the shared-memory staged
pair count (SOIL_PAIRS_STAGED=1), and every scan taken by the single-pass
kernel or by the two- and three-kernel ones (SOIL_SCAN1P_MAX), each stepped
through rebuilds on a polydisperse and a uniform-cutoff system and compared
bit for bit with the CPU oracle (state and lists, order included)."""
import os

import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import system, workloads as W

pytestmark = pytest.mark.gpu

SETTINGS = {
    "pairs-pre-off": {"SOIL_PAIRS_PRE": "0"},
    "pairs-staged": {"SOIL_PAIRS_STAGED": "1"},
    "scan-single-pass-always": {"SOIL_SCAN1P_MAX": "100000000"},
    "scan-three-kernel-always": {"SOIL_SCAN1P_MAX": "0"},
}


@pytest.mark.parametrize("name", sorted(SETTINGS))
@pytest.mark.parametrize("newton", [1, 0])
@pytest.mark.parametrize("radii", ["poly", "mono"])
def test_switch_matches_oracle(ctx, name, newton, radii):
    env = SETTINGS[name]
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        if radii == "poly":
            w = W.poly("sw", 95, 6000, 0.5, 1e-3, 0, harmonic_k=1e3, newton=newton)
        else:
            w = W.mono("sw", 96, 6000, 0.45, 1e-3, 0, harmonic_k=1e3, newton=newton)
        w.vel *= 2.0
        g, o = system.from_workload(ctx, w), oracle.from_workload(w)
        for k in range(3):
            g.step(8)
            o.step(8)
            assert_same_state(g, o, f"{name} {radii} newton={newton} step {8 * (k + 1)}")
            assert_same_lists(g, o)
        assert g.counts().rebuilds > 2
        g.close()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
