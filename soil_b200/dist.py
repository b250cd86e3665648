"""Multi-rank plumbing: one process per GPU, torch.distributed for the few
host-side exchanges the hot path needs.

Nothing on the hot path is exchanged between ranks: a single system does not
shard (every rank runs its own replica), and batched / served boxes are
independent units assigned to ranks up front.  What crosses ranks is the
barrier around the timed region, the maximum of the ranks' device times and
sums of work counters — helpers here work on NCCL (tensors on the rank's
GPU) and on gloo (CPU tensors, as the CPU tests use).
"""
import datetime
import os


def world_from_env():
    """(world, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend=None, timeout_s=300):
    """Join the process group when WORLD_SIZE > 1 (MASTER_ADDR/PORT from the
    environment).  backend None: nccl when CUDA is available, else gloo."""
    world, rank, local = world_from_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _reduce(x, op, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world):
    import torch.distributed as dist
    return x if world == 1 else _reduce(x, dist.ReduceOp.MAX, world)


def sum_over_ranks(x, world):
    import torch.distributed as dist
    return x if world == 1 else _reduce(x, dist.ReduceOp.SUM, world)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def finalize(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def lpt_partition(costs, world):
    """Greedy longest-processing-time assignment of independent units (boxes
    or jobs, cost = atoms x steps) to `world` ranks: units by decreasing
    cost, each to the currently lightest rank (ties: lowest rank).  Returns
    each rank's unit indices in ascending order; deterministic, so every
    rank computes the same plan without communicating."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
