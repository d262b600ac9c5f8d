"""Multi-GPU layout of the step: independent replicas, no data-path collective.

A single grid does not shard without an all-to-all transpose per 3D FFT, and the
batched sweep and the request stream are made of independent instances, so N
GPUs run N replicas: rank r takes the instances (or requests) whose index is
congruent to r modulo the world size, and the only collectives are the timing
and accounting reductions below (one process per GPU, torch.distributed; NCCL
on GPUs, gloo on CPU for the tests).
"""

from __future__ import annotations


def route(items: list, rank: int, world: int) -> list:
    """The share of `items` that rank `rank` of `world` runs (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return items[rank::world]


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
