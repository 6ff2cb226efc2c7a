"""Placement of independent scenes on the ranks of a job (one process per GPU).

Scenes never exchange data inside a time step, so a set of scenes shards
across GPUs with no collective on the data path: every rank builds one batch
handle (``Scene.batch``) from its own share and steps it.  The only
collectives are host-side bookkeeping — the job's time as the maximum over
ranks, and gathering per-scene results.

``assign_scenes`` balances the ranks by a per-scene cost (tets, or tets x
iterations) with the longest-processing-time rule: scenes in decreasing
cost, each to the rank with the smallest load so far (ties to the lower
rank), so the split is deterministic and every rank computes it alone.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def assign_scenes(costs: Sequence[float], world: int) -> List[List[int]]:
    """Scene indices per rank (each list ascending), balanced by cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    load = np.zeros(world)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))  # first minimum: the lowest rank among equals
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(o) for o in out]


def my_scenes(costs: Sequence[float], world: int, rank: int) -> List[int]:
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return assign_scenes(costs, world)[rank]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a float over the ranks of the default process group (the
    value itself without one).  ``device``: where the reduction buffer lives
    (a CUDA device for NCCL, None = CPU for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_by_scene(local_values: Sequence[float], mine: Sequence[int], n_scenes: int, device=None) -> np.ndarray:
    """Assemble one value per scene from every rank's share (sum-reduce of a
    zero-filled array: each scene is owned by exactly one rank)."""
    import torch
    import torch.distributed as dist
    full = torch.zeros(n_scenes, dtype=torch.float64, device=device)
    if len(mine):
        full[torch.as_tensor(list(mine), dtype=torch.long, device=device)] = torch.as_tensor(
            np.asarray(local_values, np.float64), device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(full, op=dist.ReduceOp.SUM)
    return full.cpu().numpy()
