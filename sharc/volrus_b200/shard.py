"""Sharding independent level-set grids across GPUs (one process per GPU).

A batch of uneven grids (``LevelSet.spheres``) has no data dependence between
grids, so the multi-GPU form of the batched step assigns whole grids to ranks
and runs each rank's share as one batch on its own device: no collective
touches the data path.  Only reported totals cross ranks (an FP64 sum of
active voxels and the maximum of per-rank step times), through
``torch.distributed`` with whatever backend the process group has (NCCL on
GPUs, gloo on CPU for tests).

Partitioning is greedy longest-processing-time first over a per-grid cost
estimate: grids sorted by decreasing cost (ties by index) each go to the rank
with the smallest load so far (ties by rank), so every rank computes the same
assignment from the same inputs without communicating.
"""
from __future__ import annotations

import numpy as np


def sphere_grid_cost(spheres: np.ndarray, half_width: float = 3.0) -> float:
    """Estimated band voxels of a union of spheres: sum over spheres of the
    shell volume 4 pi r^2 (2 hw) (overlaps ignored).  ``spheres``: (n, 4)
    rows (cx, cy, cz, r) in voxels."""
    s = np.asarray(spheres, np.float64).reshape(-1, 4)
    return float(np.sum(4.0 * np.pi * s[:, 3] ** 2 * (2.0 * half_width)))


def partition_lpt(costs, world: int) -> list[list[int]]:
    """Greedy LPT assignment of items to `world` ranks; returns per-rank item
    indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def imbalance(costs, parts) -> float:
    """max rank load / mean rank load (1.0 = perfect balance)."""
    costs = np.asarray(costs, np.float64)
    loads = np.array([costs[p].sum() if p else 0.0 for p in parts])
    return float(loads.max() / max(loads.mean(), 1e-300))


def reduce_totals(active_voxels: float, step_ms: float, device=None):
    """Whole-job totals across ranks: (sum of active voxels in FP64, max of
    step times).  Without an initialised process group, the local values."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(active_voxels), float(step_ms)
    a = torch.tensor([float(active_voxels)], dtype=torch.float64, device=device)
    t = torch.tensor([float(step_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(a, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(a.item()), float(t.item())


def shard_of(grids, rank: int, world: int, half_width: float = 3.0):
    """This rank's share of a list of (spheres, velocity[, ...]) grids and the
    global indices it holds."""
    costs = [sphere_grid_cost(g[0], half_width) for g in grids]
    idx = partition_lpt(costs, world)[rank]
    return [grids[i] for i in idx], idx
