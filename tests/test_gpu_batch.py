"""Batched stepping (soil_batch_*): every member is bit-identical to the same
system stepped alone with soil_step, and to the CPU oracle.

The boxes mix sizes, packing fractions, shear (sheared boxes rebuild every
step, the others only on displacement), both filter modes, Newton on and off
and a short sort period (periodic spatial sorts that find the identity and
ones that do not).  Batches are stepped in chunks that differ from the alone
runs, so the deferred final half-kick is flushed at different steps.
"""
import numpy as np
import pytest

from helpers import assert_same_lists, assert_same_state, pair
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu


def mixed_boxes(count=8, nmax=3000):
    ws = []
    for i in range(count):
        w = W.config4_box(i, nmin=256, nmax=nmax, steps=40)
        if i % 4 == 3:
            w.cfg.filter = abi.SOIL_FILTER_FP32_RECHECK
        if i % 4 == 2:
            w.cfg.sort_every = 7
        if i == 5:
            w.cfg.newton = 0
        ws.append(w)
    # a fast-sheared box whose tilt wraps inside the run, with periodic sorts
    # on top of its every-step rebuilds
    w = W.mono("fast-shear", 9, 1500, 0.4, 1e-3, 40, harmonic_k=1e3, shear_rate=5.0)
    w.cfg.sort_every = 5
    ws.append(w)
    return ws


def assert_same(a, b, what, filter_stats=True):
    assert_same_state(a, b, what)
    assert_same_lists(a, b, what)
    np.testing.assert_array_equal(a.sort_perm(), b.sort_perm(), err_msg=f"{what} sort perm")
    ca, cb = a.counts(), b.counts()
    assert ca.sorts == cb.sorts, what
    if filter_stats:  # the oracle does not count filter candidates
        assert (ca.filter_candidates, ca.filter_rechecked) == \
            (cb.filter_candidates, cb.filter_rechecked), what


def test_batch_equals_alone(ctx):
    ws = mixed_boxes()
    alone = [system.from_workload(ctx, w) for w in ws]
    mixed = [system.from_workload(ctx, w) for w in ws]
    for s in alone:
        s.step(13)
        s.step(27)
    batch = system.Batch(ctx)
    for s in mixed:
        batch.add(s)
    assert len(batch) == len(ws)
    batch.step(5)
    batch.step(1)
    batch.step(34)
    for k, (a, m) in enumerate(zip(alone, mixed)):
        assert_same(a, m, f"box {k} ({ws[k].name})")
    assert any(m.counts().rebuilds > 2 for m in mixed)
    st = batch.stats()
    assert st["steps"] == 40
    batch.close()
    for s in alone + mixed:
        s.close()


def test_batch_threaded_planning_equals_alone(ctx, monkeypatch):
    """The same boxes planned on four host threads (parallel from one box)."""
    monkeypatch.setenv("SOIL_HOST_THREADS", "4")
    monkeypatch.setenv("SOIL_HOST_MIN_PARALLEL", "1")
    ws = mixed_boxes()
    alone = [system.from_workload(ctx, w) for w in ws]
    mixed = [system.from_workload(ctx, w) for w in ws]
    for s in alone:
        s.step(31)
    batch = system.Batch(ctx)
    for s in mixed:
        batch.add(s)
    batch.step(31)
    for k, (a, m) in enumerate(zip(alone, mixed)):
        assert_same(a, m, f"box {k} ({ws[k].name})")
    batch.close()


def test_batch_fresh_boxes_ghost_growth(ctx):
    """Fresh boxes (first step in the batch) whose ghosts outgrow the first
    reservation, next to small boxes: the border pass is repeated for the
    large ones only, and every box still matches its alone run.  The first
    reservation assumes a uniform density, so the large boxes crowd 45% of
    their atoms into a column along the low x / low y edge (three images
    each: about 1.7 ghosts per atom instead of 0.35)."""
    ws = [W.poly(f"dense{i}", 11, n, 0.55, 1e-4, 10, harmonic_k=1e3, box=i)
          for i, n in enumerate([20000, 300, 24000, 280, 500, 16000])]
    for w in ws:
        if w.n >= 10000:
            col = np.arange(w.n) % 20 < 9
            w.pos[col, :2] *= 1.2 / w.L
    ws[2].shear_rate = 0.1
    alone = [system.from_workload(ctx, w) for w in ws]
    mixed = [system.from_workload(ctx, w) for w in ws]
    for s in alone:
        s.step(6)
    batch = system.Batch(ctx)
    for s in mixed:
        batch.add(s)
    batch.step(6)
    for k, (a, m) in enumerate(zip(alone, mixed)):
        assert_same(a, m, f"box {k} ({ws[k].name})")
    assert batch.stats()["border_retries"] > 0
    batch.close()


def test_batch_steady_state_allocates_nothing(ctx):
    """After the first steps, stepping (rebuilds, periodic sorts, a box's
    first displacement-triggered rebuild and sheared boxes included) takes no
    device memory: arrays are sized with headroom for drifting ghost, pair
    and bin counts, the sort's arrays follow the atom capacity, and the
    batch's staging buffers exist from its creation."""
    ws = mixed_boxes(count=8, nmax=3000)
    boxes = [system.from_workload(ctx, w) for w in ws]
    batch = system.Batch(ctx)
    for s in boxes:
        batch.add(s)
    batch.step(3)
    a0, _ = ctx.alloc_count()
    r0 = sum(s.counts().rebuilds for s in boxes)
    batch.step(60)
    a1, _ = ctx.alloc_count()
    assert sum(s.counts().rebuilds for s in boxes) > r0 + 60
    assert a1 == a0, f"{a1 - a0} device allocations in steady state"
    batch.close()
    for s in boxes:
        s.close()


def test_batch_equals_oracle(ctx):
    ws = mixed_boxes(count=4, nmax=1200)
    pairs = [pair(ctx, w) for w in ws]
    batch = system.Batch(ctx)
    for g, _ in pairs:
        batch.add(g)
    batch.step(25)
    for k, (g, o) in enumerate(pairs):
        o.step(25)
        assert_same(g, o, f"box {k} ({ws[k].name})", filter_stats=False)
    batch.close()


def test_batch_membership_changes(ctx):
    """Boxes join and leave between steps (the served loop's pattern); each
    box's result only depends on its own step count."""
    ws = mixed_boxes(count=6, nmax=2000)
    sched = {0: (0, 30), 1: (0, 12), 2: (5, 30), 3: (12, 30), 4: (5, 22), 5: (0, 30)}
    mixed = [system.from_workload(ctx, w) for w in ws]
    batch = system.Batch(ctx)
    t = 0
    for edge in (5, 12, 22, 30):
        for k, (t0, t1) in sched.items():
            if t0 == t:
                batch.add(mixed[k])
            if t1 == t:
                batch.remove(mixed[k])
        batch.step(edge - t)
        t = edge
    for k, (t0, t1) in sched.items():
        if t1 == t:
            batch.remove(mixed[k])
    assert len(batch) == 0
    for k, (t0, t1) in sched.items():
        a = system.from_workload(ctx, ws[k])
        a.step(t1 - t0)
        assert_same(a, mixed[k], f"box {k}")
        a.close()
    batch.close()


def test_batch_leave_and_rejoin(ctx):
    """A box that leaves the batch mid-run, steps alone and joins again (the
    served loop steps a lone job through the single-system path) ends bit for
    bit where it would alone, and so do the boxes that stayed."""
    ws = mixed_boxes(count=3, nmax=2000)
    boxes = [system.from_workload(ctx, w) for w in ws]
    batch = system.Batch(ctx)
    for b in boxes:
        batch.add(b)
    batch.step(7)
    batch.remove(boxes[0])
    boxes[0].step(9)
    batch.step(9)
    batch.add(boxes[0])
    batch.step(6)
    for b in boxes:
        batch.remove(b)
    for k, w in enumerate(ws):
        a = system.from_workload(ctx, w)
        a.step(22)
        assert_same(a, boxes[k], f"box {k}")
        a.close()
    batch.close()


def test_batch_rejects_unsupported(ctx):
    w = W.config1(n=1024, steps=10)  # no consumer
    s = system.from_workload(ctx, w)
    batch = system.Batch(ctx)
    with pytest.raises(abi.SoilError):
        batch.add(s)
    # a member steps only through its batch; once removed it steps alone
    m = system.from_workload(ctx, W.config4_box(0, nmin=256, nmax=1000, steps=5))
    batch.add(m)
    with pytest.raises(abi.SoilError):
        m.step(1)
    batch.step(2)
    batch.remove(m)
    m.step(1)
    assert m.counts().step == 3
    batch.close()
    s.close()
    m.close()
