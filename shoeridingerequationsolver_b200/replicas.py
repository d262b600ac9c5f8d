"""Multi-GPU layout of the step: independent replicas, no data-path collective.

A single grid does not shard without an all-to-all transpose per 3D FFT, and the
batched sweep and the request stream are made of independent instances, so N
GPUs run N replicas: rank r takes its share of the instances (balanced by grid
points) or of the requests (round robin), and the only collectives are the
timing and accounting reductions below (one process per GPU, torch.distributed; NCCL
on GPUs, gloo on CPU for the tests).
"""

from __future__ import annotations


def route(items: list, rank: int, world: int) -> list:
    """The share of `items` that rank `rank` of `world` runs (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return items[rank::world]


def route_balanced(items: list, rank: int, world: int, weight) -> list:
    """The share of `items` that rank `rank` runs when every rank should get the
    same total weight (grid points of the instances): largest first, each to the
    least loaded rank (ties to the lowest rank).  Every rank computes the same
    assignment from the same list, so no exchange is needed."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(items)), key=lambda i: (-weight(items[i]), i))
    load = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += weight(items[i])
        if r == rank:
            mine.append(i)
    return [items[i] for i in sorted(mine)]


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """Slowest rank's value (timings are reported as the max over ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """Whole-job total of a per-rank count (grid points x steps, requests)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
