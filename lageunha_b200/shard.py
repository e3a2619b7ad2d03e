"""Sharding independent boxes over ranks (one GPU per rank).

An ensemble or a stream of served requests splits by box: every box is
evaluated on exactly one rank and no data crosses ranks, so the only
collectives are the host-side reductions of timings and metrics. Boxes go to
ranks by longest-processing-time-first on the cost Np log2 Np (the sort and
the tree walk both grow that way), which keeps the busiest rank within 4/3
of the optimum.
"""
from __future__ import annotations

import heapq
import math


def box_cost(np_: int) -> float:
    return float(np_) * math.log2(max(np_, 2))


def assign_boxes(sizes, nranks: int) -> list[list[int]]:
    """Indices of the boxes each rank evaluates (LPT on box_cost), every box
    on exactly one rank; within a rank the boxes keep their input order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-box_cost(sizes[i]), i))
    heap = [(0.0, r) for r in range(nranks)]
    heapq.heapify(heap)
    out = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + box_cost(sizes[i]), r))
    return [sorted(x) for x in out]


def rank_loads(sizes, assignment) -> list[float]:
    return [sum(box_cost(sizes[i]) for i in boxes) for boxes in assignment]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest of every rank's value (a timing): an all-reduce when a
    process group is up, the value itself otherwise."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
