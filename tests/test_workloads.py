"""Seeded generators: deterministic bytes, documented shapes and ranges."""
import math

import numpy as np

from soil_b200 import workloads as W


def test_generators_are_deterministic():
    a, b = W.config1(n=1000), W.config1(n=1000)
    assert a.pos.tobytes() == b.pos.tobytes() and a.vel.tobytes() == b.vel.tobytes()
    c = W.poly("x", 99, 1000, 0.5, 1e-4, 1)
    d = W.poly("x", 99, 1000, 0.5, 1e-4, 1)
    assert c.radius.tobytes() == d.radius.tobytes()


def test_config1_box_and_velocities():
    w = W.config1()
    assert w.n == 32768
    assert abs(w.L - (32768 * math.pi / 6 / 0.30) ** (1 / 3)) < 1e-12
    assert np.all((w.pos >= 0) & (w.pos < w.L))
    assert np.max(np.abs(w.vel.mean(axis=0))) < 1e-12
    assert abs(w.vel.std() - 1.0) < 0.02
    assert w.cfg.skin_fraction == 1.1 and np.all(w.cutoff == 0.5)


def test_poly_packing_fraction_and_skin():
    w = W.poly("p", 2, 20000, 0.5, 1e-4, 1)
    assert np.all((w.radius >= 0.4) & (w.radius <= 0.6))
    phi = np.sum(4 / 3 * math.pi * w.radius ** 3) / w.L ** 3
    assert abs(phi - 0.5) < 1e-12
    assert np.allclose(w.cutoff, w.radius + 0.05)
    assert w.cfg.additive_skin == 0.1 and w.cfg.skin_fraction == 1.0


def test_batched_and_served_ranges():
    ns = [W.config4_box(i, steps=1).n for i in range(64)]
    assert min(ns) >= 256 and max(ns) <= 65536
    j = W.config5_job(3)
    assert 1024 <= j.n <= 262144 and 500 <= j.steps <= 5000 and 0 <= j.shear_rate <= 0.2
