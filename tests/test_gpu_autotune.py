"""The autotuner on the GPU: it picks a bin size per size class by timing
(soil_b200.autotune.tune), and a tuned configuration gives the same bits
alone, batched and in the CPU oracle (with the same bin size)."""
import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import autotune, system, workloads as W

pytestmark = pytest.mark.gpu


def test_tuned_boxes_identical_alone_batched_and_oracle(ctx):
    ws = [W.config4_box(i, steps=0) for i in (0, 1, 2, 3)]
    samples = {}
    for w in ws:
        samples.setdefault(autotune.size_class(w.n), []).append(w)
    table = autotune.tune(ctx, samples, steps=4, warmup=2)
    assert set(table.entries) == {str(c) for c in samples}
    for e in table.entries.values():
        assert e["bin_factor"] in autotune.CANDIDATES and e["rate"] > 0
    ws = [table.apply(w) for w in ws]
    alone = [system.from_workload(ctx, w) for w in ws]
    for s in alone:
        s.step(12)
    batched = [system.from_workload(ctx, w) for w in ws]
    b = system.Batch(ctx)
    for s in batched:
        b.add(s)
    b.step(12)
    for w, a, s in zip(ws, alone, batched):
        assert_same_state(a, s, w.name)
        assert_same_lists(a, s, w.name)
    o = oracle.from_workload(ws[0])
    o.step(12)
    assert_same_state(alone[0], o)
    assert_same_lists(alone[0], o)
    b.close()
