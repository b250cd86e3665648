"""Multi-rank host logic on CPU: two gloo ranks (spawned processes, rendezvous
on 127.0.0.1) exercise the reductions and barrier bench.py uses around its
timed region, the rank-independent work partition, and host-side failure
detection: a rank that leaves makes the other's next collective fail within
the process-group timeout instead of hanging."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from soil_b200 import dist, workloads


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))


def _reduce_worker(rank, world, port, q):
    _env(rank, world, port)
    w, r, _ = dist.init(backend="gloo", timeout_s=30)
    dist.barrier(w)
    mx = dist.max_over_ranks(10.0 * (r + 1), w)
    sm = dist.sum_over_ranks(r + 1, w)
    costs = [workloads.config4_size(i) for i in range(64)]
    part = dist.lpt_partition(costs, w)
    q.put((r, mx, sm, part[r]))
    dist.finalize(w)


def _leaving_worker(rank, world, port, q):
    _env(rank, world, port)
    w, r, _ = dist.init(backend="gloo", timeout_s=3)
    dist.barrier(w)
    if r == 1:
        q.put((r, "left"))
        q.close()
        q.join_thread()  # the message is out before the process ends
        os._exit(0)  # leaves between steps, with nothing in flight
    try:
        dist.max_over_ranks(1.0, w)
        q.put((r, "no error"))
    except Exception as e:  # the collective fails instead of hanging
        q.put((r, "error: " + type(e).__name__))
    q.close()
    q.join_thread()
    os._exit(0)


def _run(target, world=2, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=timeout)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_two_rank_reductions_and_partition():
    out = _run(_reduce_worker)
    assert [o[1] for o in out] == [20.0, 20.0]
    assert [o[2] for o in out] == [3.0, 3.0]
    parts = [o[3] for o in out]
    assert sorted(parts[0] + parts[1]) == list(range(64))  # every box on exactly one rank
    costs = [workloads.config4_size(i) for i in range(64)]
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)  # LPT bound: within one unit


def test_rank_that_leaves_is_detected():
    out = _run(_leaving_worker, timeout=90)
    assert out[1] == (1, "left")
    assert out[0][1].startswith("error"), out


def test_lpt_partition_is_deterministic_and_single_rank_identity():
    costs = [5, 3, 8, 8, 1, 2]
    assert dist.lpt_partition(costs, 1) == [list(range(6))]
    a = dist.lpt_partition(costs, 3)
    assert a == dist.lpt_partition(costs, 3)
    assert sorted(sum(a, [])) == list(range(6))
    # largest first, ties to the lowest rank: 8 -> r0, 8 -> r1, 5 -> r2, 3 -> r2, 2 -> r0/r1...
    assert 2 in a[0] and 3 in a[1] and 0 in a[2]


@pytest.mark.parametrize("world", [1])
def test_single_process_helpers_are_identity(world):
    assert dist.max_over_ranks(3.5, world) == 3.5
    assert dist.sum_over_ranks(2.0, world) == 2.0
    dist.barrier(world)
