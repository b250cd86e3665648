"""Registered AtomData columns of every flag class against the CPU oracle, bit
for bit, checked every few steps across sorts, border passes and reverse folds
(crates/soil_core/src/atom.rs:163-377 and the derive's fan-out,
crates/soil_derive/src/lib.rs:392-500):

  orient  width 3, #[forward]: a consumer adds to the locals' values; ghosts
          must hold their owner's value (forward comm, borders);
  torque  width 2, #[reverse]: a consumer adds to every atom's value; ghost
          values fold into their owners after the force phase;
  zacc    width 1, #[zero]: cleared with the forces every step, then written;
  label   width 2, unflagged: only permuted by the sort and copied to new
          ghosts.

The consumer is tests/hooks/registry_hook.cu on the GPU (through the
force-hook ABI, which also exercises the view's column layout
columns[c][k * stride + i]) and the oracle's column probe on the CPU."""
import os
import sys

import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state, attach_registry_hook, build_hook
from soil_b200 import abi, system, workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import REGISTRY_COLUMNS, REGISTRY_PROBE  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def registry_lib(tmp_path_factory):
    return build_hook(tmp_path_factory.mktemp("hook"), "registry_hook")


def _make(sysmake, w):
    s = sysmake(w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    data = [w.radius]
    for k, (name, width, flags) in enumerate(REGISTRY_COLUMNS):
        s.register_column(name, width, flags)
        data.append(np.stack([W.uniform(w.seed, 0, 70 + 4 * k + c, w.n) for c in range(width)],
                             axis=1).reshape(w.n, width))
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=data)
    s.set_harmonic(w.harmonic_k, rc)
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    s.setup()
    return s


@pytest.mark.parametrize("shear", [0.0, 1.0])
def test_registered_columns_match_the_oracle(ctx, registry_lib, shear):
    w = W.poly("registry", 71, 3000, 0.45, 1e-3, 0, harmonic_k=1e3, shear_rate=shear)
    w.vel *= 3.0
    g = _make(lambda b, c, dt: system.System(ctx, b, c, dt), w)
    attach_registry_hook(registry_lib, w.harmonic_k)(g, REGISTRY_PROBE)
    o = _make(oracle.OracleSystem, w)
    o.set_column_probe(**REGISTRY_PROBE)
    widths = [1] + [c[1] for c in REGISTRY_COLUMNS]
    for k in range(5):
        g.step(8)
        o.step(8)
        what = f"after {8 * (k + 1)} steps"
        assert_same_state(g, o, what)  # compares every column bit for bit
        assert_same_lists(g, o, what)
        for c, width in enumerate(widths):
            assert g.column(c).shape == (g.counts().nlocal + g.counts().nghost, width)
    c = g.counts()
    assert c.rebuilds > 5 and c.nghost > 0
    # the flags did what they say: ghosts hold their owner's unflagged values
    # (forward values lag by this step's write to the locals, which comes
    # after forward comm); the zero column holds this step's write only
    a = g.atoms()
    nl = c.nlocal
    zacc, label = g.column(3), g.column(4)
    owner = np.empty(c.nlocal + c.nghost, np.int64)
    owner[:nl] = np.arange(nl)
    for gi in range(nl, nl + c.nghost):  # follow origins down to the local owner
        q = a["origin"][gi]
        while q >= nl:
            q = a["origin"][q]
        owner[gi] = q
    np.testing.assert_array_equal(label[nl:], label[owner[nl:]])
    np.testing.assert_array_equal(zacc[:nl, 0], 0.25 * a["pos"][:nl, 0])
    g.close()
