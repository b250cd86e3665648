"""Host-side pieces of the served benchmark: the seeded Poisson arrival
stream and the FIFO latency model of the plain one-job-at-a-time path."""
import numpy as np

from soil_b200 import serve


def test_poisson_arrivals_rate_and_determinism():
    a = serve.poisson_arrivals(4.0, 20000, seed=5)
    b = serve.poisson_arrivals(4.0, 20000, seed=5)
    np.testing.assert_array_equal(a, b)
    assert a[0] == 0.0 and np.all(np.diff(a) >= 0)
    gaps = np.diff(a)
    assert abs(gaps.mean() - 0.25) < 0.01          # mean gap 1/rate
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.03  # exponential: CV = 1


def test_fifo_latencies_lindley():
    arr = np.array([0.0, 1.0, 1.5, 10.0])
    svc = np.array([2.0, 2.0, 1.0, 0.5])
    lat = serve.fifo_latencies(arr, svc)
    # job 0: 0->2; job 1 starts 2 ends 4; job 2 starts 4 ends 5; job 3 starts 10
    np.testing.assert_allclose(lat, [2.0, 3.0, 3.5, 0.5])
