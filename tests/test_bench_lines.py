"""The committed bench lines (profiles/bench_*_line.json) are internally
consistent: each roofline's achieved bandwidth is its algorithmic bytes per
launch over the mean launch time, its fraction is achieved over the stated
peak, the line's value matches its per-step time where both are given, and no
line was taken under a thermal or hardware slowdown."""
import glob
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LINES = sorted(glob.glob(os.path.join(ROOT, "profiles", "bench_*_line.json")))
BAD_REASONS = {"hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"}


def load(path):
    with open(path) as f:
        return json.load(f)


def test_lines_exist():
    names = {os.path.basename(p) for p in LINES}
    for c in ("c1", "c2", "c3", "c4", "c5", "ref"):
        assert f"bench_{c}_line.json" in names


@pytest.mark.parametrize("path", LINES, ids=os.path.basename)
def test_line_consistent(path):
    d = load(path)
    assert d["metric"] == "atom-steps/s" and d["unit"] == "atom-steps/s"
    assert d["higher_is_better"] is True
    assert d["value"] > 0
    roof = d.get("roofline")
    if roof and roof.get("algorithmic_bytes_per_launch") and roof.get("mean_launch_ms"):
        gbs = roof["algorithmic_bytes_per_launch"] / (roof["mean_launch_ms"] * 1e-3) / 1e9
        assert roof["achieved"] == pytest.approx(gbs, rel=1e-6)
        assert roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"], rel=1e-6)
        assert roof["unit"] == "GB/s" and roof["bound"] == "hbm"
    clocks = d.get("clocks")
    if clocks:
        assert not BAD_REASONS & set(clocks.get("reasons", [])), clocks
    if d.get("ms_per_step") and d.get("config", {}).get("n_atoms") and d.get("impl") != "reference":
        n = d["config"]["n_atoms"] * d.get("n_gpus", 1)
        assert d["value"] == pytest.approx(n / (d["ms_per_step"] * 1e-3), rel=1e-3)
