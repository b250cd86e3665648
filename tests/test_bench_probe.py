"""bench.py's rebuild probe separates the light and the rebuild step costs:
on a stand-in system whose chunk times follow a known model (a light-step
cost, an extra cost per rebuild and a per-call cost), the least-squares fit
recovers both costs, and an every-step-rebuild system reports its mean
rebuild step.  CPU only: the CUDA events are replaced by a model clock."""
import types

import pytest
import torch

import bench


class ModelClock:
    now = 0.0


class ModelEvent:
    def __init__(self, enable_timing=True):
        self.t = None

    def record(self, stream=None):
        self.t = ModelClock.now

    def elapsed_time(self, other):
        return other.t - self.t


class ModelSystem:
    """Light steps cost `light` ms, a rebuild step `light + extra`, and each
    step() call `per_call` more; every `period`-th step rebuilds."""

    def __init__(self, light, extra, per_call, period):
        self.light, self.extra, self.per_call, self.period = light, extra, per_call, period
        self.k = 0
        self.rebuilds = 0

    def counts(self):
        return types.SimpleNamespace(rebuilds=self.rebuilds)

    def step(self, n):
        ms = self.per_call
        for _ in range(n):
            self.k += 1
            ms += self.light
            if self.k % self.period == 0:
                self.rebuilds += 1
                ms += self.extra
        ModelClock.now += ms

    def sync(self):
        pass


@pytest.fixture
def model_events(monkeypatch):
    monkeypatch.setattr(torch.cuda, "Event", ModelEvent)
    ModelClock.now = 0.0


@pytest.mark.parametrize("period", [7, 11, 15])
def test_probe_separates_light_and_rebuild(model_events, period):
    s = ModelSystem(light=0.36, extra=1.14, per_call=0.05, period=period)
    out = bench.rebuild_probe(s, stream=None)
    assert out["rebuilds"] >= 3
    assert out["ms_per_light_step"] == pytest.approx(0.36, rel=1e-9)
    assert out["ms_per_rebuild_step"] == pytest.approx(1.50, rel=1e-9)
    rate = out["rebuilds"] / out["steps"]
    assert out["ms_per_step_at_rebuild_rate"] == pytest.approx(0.36 + rate * 1.14, rel=1e-9)


def test_probe_every_step_rebuilds(model_events):
    s = ModelSystem(light=0.1, extra=0.34, per_call=0.0, period=1)
    out = bench.rebuild_probe(s, stream=None)
    assert out["rebuild_rate"] == 1.0
    assert out["ms_per_light_step"] is None
    assert out["ms_per_rebuild_step"] == pytest.approx(0.44, rel=1e-9)
