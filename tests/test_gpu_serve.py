"""Served mode (soil_server_*): jobs that arrive while others run are
admitted as memory and slots free up, advanced together, and each job's
result is bit-identical to the same job run alone through soil_step."""
import time

import numpy as np
import pytest

from soil_b200 import abi, serve, system, workloads as W

pytestmark = pytest.mark.gpu


def small_jobs(count, nmax=5000, smin=20, smax=90):
    return [W.config5_job(i, nmin=1024, nmax=nmax, smin=smin, smax=smax) for i in range(count)]


def alone_result(ctx, w):
    s = system.from_workload(ctx, w)
    s.step(w.steps)
    a = s.atoms(local_only=True)
    s.close()
    return a


def assert_same_result(r, a, what):
    np.testing.assert_array_equal(r["tag"], a["tag"], err_msg=f"{what} tag")
    np.testing.assert_array_equal(r["image"], a["image"], err_msg=f"{what} image")
    for k in ("pos", "vel"):
        np.testing.assert_array_equal(r[k].view(np.uint64), a[k].view(np.uint64),
                                      err_msg=f"{what} {k}")


def test_served_jobs_equal_alone(ctx):
    ws = small_jobs(7)
    sctx = system.Context(0)
    sv = serve.Server(sctx, quantum_steps=16)
    # two waves: the second arrives while the first runs and joins it at the
    # next admission point (a lone job steps through the single-system path,
    # so arrivals far apart would each run alone)
    ids = [sv.submit(w) for w in ws[:4]]
    time.sleep(0.002)
    ids += [sv.submit(w) for w in ws[4:]]
    infos = [sv.wait(j, timeout=300) for j in ids]
    assert all(i["state"] == "done" for i in infos), infos
    st = sv.stats()
    assert st["completed"] == len(ws) and st["max_active"] >= 2
    results = [sv.result(j) for j in ids]
    sv.close()
    sctx.close()
    for k, (w, r) in enumerate(zip(ws, results)):
        assert_same_result(r, alone_result(ctx, w), f"job {k} ({w.name}, {w.steps} steps)")


def test_served_admission_respects_budget(ctx):
    ws = small_jobs(4, nmax=3000, smax=40)
    sctx = system.Context(0)
    # room for one job's reservation at a time
    per_atom, per_job = 1024, 1 << 20
    budget = max(w.n for w in ws) * per_atom + per_job
    sv = serve.Server(sctx, hbm_budget_bytes=budget, bytes_per_atom=per_atom,
                      bytes_per_job=per_job, quantum_steps=8)
    ids = [sv.submit(w) for w in ws]
    infos = [sv.wait(j, timeout=300) for j in ids]
    assert all(i["state"] == "done" for i in infos)
    st = sv.stats()
    assert st["max_active"] == 1 and st["reserved_bytes"] == 0
    # first come first served: each job is admitted after the previous finished
    for a, b in zip(infos, infos[1:]):
        assert b["t_admit"] >= a["t_done"] - 1e-6
    results = [sv.result(j) for j in ids]
    sv.close()
    sctx.close()
    for k, (w, r) in enumerate(zip(ws, results)):
        assert_same_result(r, alone_result(ctx, w), f"job {k}")


def test_served_cancel_and_release(ctx):
    ws = small_jobs(2, nmax=2000, smin=4000, smax=5000)
    sctx = system.Context(0)
    sv = serve.Server(sctx, quantum_steps=10)
    a = sv.submit(ws[0])
    b = sv.submit(ws[1])
    sv.cancel(b)
    time.sleep(0.2)
    sv.cancel(a)
    ia, ib = sv.wait(a, timeout=120), sv.wait(b, timeout=120)
    assert ia["state"] == "cancelled" and ib["state"] == "cancelled"
    with pytest.raises(abi.SoilError):
        sv.result(a)
    sv.release(a)
    with pytest.raises(abi.SoilError):
        sv.poll(a)
    sv.close()
    sctx.close()


def test_served_failures_are_isolated(ctx):
    """Host-side fault injection: a malformed request is refused at submit;
    a job that does not fit the context's HBM budget fails with an error
    message and frees what it took; the loop goes on serving."""
    sctx = system.Context(0, hbm_budget_bytes=64 << 20)
    sv = serve.Server(sctx, quantum_steps=8)
    bad = W.config5_job(0, nmin=1024, nmax=2000, smin=20, smax=30)
    bad.harmonic_k = 0.0  # no consumer: not a servable job
    with pytest.raises(abi.SoilError):
        sv.submit(bad)
    big = W.config5_job(1, nmin=200000, nmax=262144, smin=20, smax=30)
    small = W.config5_job(2, nmin=1024, nmax=2000, smin=20, smax=30)
    jb = sv.submit(big)
    js = sv.submit(small)
    ib, is_ = sv.wait(jb, timeout=120), sv.wait(js, timeout=120)
    assert ib["state"] == "failed" and "budget" in sv.error(jb)
    assert is_["state"] == "done"
    assert_same_result(sv.result(js), alone_result(ctx, small), "job after a failure")
    sv.close()
    assert sctx.bytes_in_use() < (64 << 20)
    sctx.close()
