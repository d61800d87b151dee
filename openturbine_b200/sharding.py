"""Placement of independent models on ranks (one process per GPU).

Models never share nodes or constraints with each other, so a time step needs
no data exchange between GPUs: each rank advances the models it owns, and the
only collectives are the timing / counting reductions of the benchmark and an
optional end-of-run gather of per-model results.  This module holds that host
logic so it can be tested with CPU process groups.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def beam_cost(num_nodes: int, num_qp: int) -> float:
    """Relative cost of one Newton iteration of a beam element: the node-pair
    integration (N^2 Q) and the dense LU of the 6N-sized system."""
    n = 6 * num_nodes
    return 410.0 * num_nodes * num_nodes * num_qp + (2.0 / 3.0) * n ** 3


def partition(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of models to ranks.

    Deterministic: every rank computes the same partition from the same costs.
    Returns, per rank, the model indices in ascending order."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    parts: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def weak_shard_first_id(rank: int, models_per_rank: int) -> int:
    """First model id of a rank's own batch when every rank gets a fresh batch
    of the same size (weak scaling)."""
    return rank * models_per_rank


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar (the timed region of the slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """Sum of a per-rank scalar (units processed by the whole job)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return float(t.item())
