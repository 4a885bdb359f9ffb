"""Replicas and jobs across GPUs: independent units (batch replicas, served
jobs) are split over the ranks by a size-balanced greedy rule, and only
metrics cross ranks afterwards; nothing is exchanged on the data path."""
from __future__ import annotations

from typing import List, Sequence


def balanced_partition(sizes: Sequence[float], nranks: int) -> List[List[int]]:
    """Unit indices for each rank: largest unit first, each to the rank with
    the least total so far (ties to the lower rank); within a rank the units
    keep their original order.  Deterministic, so every rank computes the same
    split without communicating.  The largest rank total exceeds the mean by
    at most the largest unit."""
    if nranks < 1:
        raise ValueError("nranks must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-float(sizes[i]), i))
    load = [0.0] * nranks
    parts: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(sizes[i])
    return [sorted(p) for p in parts]


def sum_over_ranks(value: float, dist, device=None) -> float:
    """Sum of a per-rank number (units processed) over the ranks."""
    if not dist:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_objects(obj, dist):
    """Every rank's `obj` (small metric records) on every rank, in rank order."""
    if not dist:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
