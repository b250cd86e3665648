"""The per-size-class bin-size table (soil_b200.autotune): classes, lookup,
application to a workload's configuration, and its JSON round trip (CPU)."""
import pytest

from soil_b200 import autotune, workloads as W


def test_size_classes():
    assert [autotune.size_class(n) for n in (1, 2, 3, 255, 256, 65535, 65536)] == \
        [0, 1, 1, 7, 8, 15, 16]


def test_table_applies_and_round_trips(tmp_path):
    t = autotune.Table({8: {"bin_factor": 1.5, "rate": 1.0}, "12": {"bin_factor": 2.0, "rate": 2.0}})
    w_small = W.poly("t8", 1, 300, 0.4, 1e-4, 0)      # class 8
    w_big = W.poly("t12", 2, 5000, 0.4, 1e-4, 0)      # class 12
    w_none = W.poly("t10", 3, 1500, 0.4, 1e-4, 0)     # class 10: not tuned
    # the largest pair cutoff: 2 * max(r + skin/2) * skin_fraction
    assert autotune.max_pair_cutoff(w_small) == 2.0 * float(w_small.cutoff.max())
    assert t.apply(w_small).cfg.bin_size == 1.5 * autotune.max_pair_cutoff(w_small)
    assert t.apply(w_big).cfg.bin_size == 2.0 * autotune.max_pair_cutoff(w_big)
    before = w_none.cfg.bin_size
    assert t.apply(w_none).cfg.bin_size == before
    p = tmp_path / "sub" / "table.json"
    t.save(str(p))
    u = autotune.Table.load(str(p))
    assert u.entries == t.entries
    assert u.factor(300) == 1.5 and u.factor(1500) is None


def test_table_refuses_unknown_version(tmp_path):
    p = tmp_path / "t.json"
    p.write_text('{"version": 7, "classes": {}}')
    with pytest.raises(ValueError):
        autotune.Table.load(str(p))
