"""A single system whose ghosts outgrow the first reservation on its first
build.  soil_step reads the border pass's totals back only at the neighbor
build's synchronisation, so the overflow is found after the build's first
kernels ran on a partial ghost set; the arrays then grow and the pass and
the build are repeated.  The result must still be the oracle's, bit for bit.
The first reservation assumes a uniform density; here 45% of the atoms are
crowded into a column along the low x / low y edge (three images each), the
same crowding that makes a batch repeat its border pass
(tests/test_gpu_batch.py)."""
import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import system, workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shear", [0.0, 0.1])
def test_first_build_ghost_overflow_matches_oracle(ctx, shear):
    w = W.poly("dense", 11, 20000, 0.55, 1e-4, 0, harmonic_k=1e3)
    col = np.arange(w.n) % 20 < 9
    w.pos[col, :2] *= 1.2 / w.L
    w.shear_rate = shear
    g, o = system.from_workload(ctx, w), oracle.from_workload(w)
    for k in range(3):
        g.step(2)
        o.step(2)
        assert_same_state(g, o, f"shear={shear} step {2 * (k + 1)}")
        assert_same_lists(g, o)
    c = g.counts()
    assert c.nghost > 1.0 * c.nlocal  # far above the uniform-density reservation
    g.close()
