"""Every kernel of the built-in consumer (SOIL_FORCE: the per-atom gather with
a separate reverse pass, the per-root walk over the CSR and its transpose,
and over grouped sequences warp tiles with 4 or 2 rows per chunk or one root
per thread) gives the reference's forces bit for bit: single systems with newton
on and off against the CPU oracle, and batched boxes against the same boxes
alone."""
import os

import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import system, workloads as W

pytestmark = pytest.mark.gpu

VARIANTS = ["gather", "csr", "tiles4", "tiles2", "walk"]


@pytest.fixture
def variant_env(request):
    old = os.environ.get("SOIL_FORCE")
    os.environ["SOIL_FORCE"] = request.param
    yield request.param
    if old is None:
        del os.environ["SOIL_FORCE"]
    else:
        os.environ["SOIL_FORCE"] = old


@pytest.mark.parametrize("variant_env", VARIANTS, indirect=True)
@pytest.mark.parametrize("newton", [1, 0])
def test_consumer_variant_matches_oracle(ctx, variant_env, newton):
    w = W.poly("fv", 91, 4000, 0.5, 1e-3, 0, harmonic_k=1e3, newton=newton)
    w.vel *= 2.0
    g, o = system.from_workload(ctx, w), oracle.from_workload(w)
    for k in range(3):
        g.step(10)
        o.step(10)
        assert_same_state(g, o, f"{variant_env} newton={newton} step {10 * (k + 1)}")
        assert_same_lists(g, o)
    assert g.counts().rebuilds > 2
    g.close()


@pytest.mark.parametrize("variant_env", VARIANTS, indirect=True)
def test_consumer_variant_batched_equals_alone(ctx, variant_env):
    ws = [W.config4_box(i, steps=0) for i in (4, 5, 6)]
    alone = [system.from_workload(ctx, w) for w in ws]
    for s in alone:
        s.step(15)
    boxes = [system.from_workload(ctx, w) for w in ws]
    b = system.Batch(ctx)
    for s in boxes:
        b.add(s)
    b.step(15)
    for w, a, s in zip(ws, alone, boxes):
        assert_same_state(a, s, f"{variant_env} {w.name}")
        assert_same_lists(a, s, w.name)
    b.close()


@pytest.mark.parametrize("order", ["1", "0"])
def test_fused_forward_and_root_order_match_oracle(ctx, order):
    """Forward comm inside the integration pass (SOIL_FWD_FUSED=1) and the CSR
    walk with and without its per-block root order give the reference's bits."""
    keys = ("SOIL_FWD_FUSED", "SOIL_ROOT_ORDER", "SOIL_RESIDENT_STEPS", "SOIL_FORCE")
    old = {k: os.environ.get(k) for k in keys}
    os.environ.update({"SOIL_FWD_FUSED": "1", "SOIL_ROOT_ORDER": order,
                       "SOIL_RESIDENT_STEPS": "0", "SOIL_FORCE": "csr"})
    try:
        w = W.poly("ff", 92, 4000, 0.5, 1e-3, 0, harmonic_k=1e3)
        w.vel *= 2.0
        g, o = system.from_workload(ctx, w), oracle.from_workload(w)
        g.step(30)
        o.step(30)
        assert_same_state(g, o)
        assert_same_lists(g, o)
        g.close()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


class _Dev:
    """A device array as __cuda_array_interface__, for torch.as_tensor."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3}


def _grow_radius_through_view(g, atoms, factor):
    import torch
    v = g.view()
    cols = torch.as_tensor(_Dev(v.columns, v.ncolumns, "<u8"), device="cuda").cpu()
    rad = torch.as_tensor(_Dev(int(cols[0]), v.nlocal, "<f8"), device="cuda")
    rad[atoms] *= factor
    torch.cuda.synchronize()


@pytest.mark.parametrize("force", ["csr", "walk"])
@pytest.mark.parametrize("resident", ["1", "0"])
def test_packed_records_follow_view_writes(ctx, force, resident):
    """The consumer kernels read packed (x, y, z, r) records that the
    integration pass and forward comm keep current; radii written through a
    device view between steps must reach them.  Packed and column reads give
    the same bits before and after such a write."""
    keys = ("SOIL_PACKED", "SOIL_FORCE", "SOIL_RESIDENT_STEPS")
    old = {k: os.environ.get(k) for k in keys}
    try:
        runs = []
        for packed in ("1", "0"):
            os.environ.update({"SOIL_PACKED": packed, "SOIL_FORCE": force,
                               "SOIL_RESIDENT_STEPS": resident})
            w = W.poly("pk", 93, 4000, 0.5, 1e-4, 0, harmonic_k=1e3)
            g = system.from_workload(ctx, w)
            g.step(12)
            _grow_radius_through_view(g, [3, 500, 2100, 3999], 1.05)
            g.step(12)
            runs.append(g)
        assert_same_state(runs[0], runs[1], f"{force} resident={resident}")
        assert_same_lists(runs[0], runs[1])
        for g in runs:
            g.close()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
