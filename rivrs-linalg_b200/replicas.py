"""Host logic of runs on several GPUs of one node (one process per GPU).

The single-system numeric phase does not shard (the top of the assembly tree
is a serial chain of large fronts), so several GPUs either run independent
replicas of the same workload or, for many independent systems, split the
systems between them: no collective touches the data path.  torch.distributed
serves only the barrier and the max-over-ranks of the timings.
"""
from __future__ import annotations


def shard(weights, rank: int, world: int) -> list:
    """Indices of the items rank `rank` of `world` takes: the largest items
    first, each to the rank with the least total weight so far (ties to the
    lower rank), so every item has exactly one rank and the totals balance.
    Returned in increasing index order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += float(weights[i])
    return [i for i in range(len(weights)) if owner[i] == rank]


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The largest `value` over the ranks of the default process group (the
    value itself without one): a job's time is its slowest rank's."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The sum of `value` over the ranks (work done by the whole job)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
