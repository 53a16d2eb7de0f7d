"""Sharding independent simulations across GPUs (one process per GPU).

Simulations in a batch or a request stream never exchange data, so N GPUs
split them with no data-path collective: every rank computes the same
assignment from the same list of footprints (device bytes, a proxy for the
work per step) and keeps its own share.  The only collectives are on the
host side of the measurement: a barrier around the timed region and the
max-over-ranks of the elapsed times.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def assign(weights: Sequence[float], world: int) -> List[List[int]]:
    """Items per rank, longest-processing-time first: items in descending
    weight order (ties by index) each go to the rank with the least load so
    far (ties by rank).  Deterministic, so every rank gets the same answer."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    for r in range(world):
        out[r].sort()
    return out


def my_share(weights: Sequence[float], rank: int, world: int) -> List[int]:
    return assign(weights, world)[rank]


def imbalance(weights: Sequence[float], world: int) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    loads = [sum(float(weights[i]) for i in part) for part in assign(weights, world)]
    mean = sum(loads) / max(world, 1)
    return max(loads) / mean if mean > 0 else 1.0


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest ``value`` over all ranks of the default process group
    (the value itself without one)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
