"""Sharding of independent boxes across ranks (one process per GPU).

Ensembles and served jobs are sets of independent boxes: a multi-GPU run
gives each rank a share of the boxes and advances it with one batch
(jt_batch_* on that rank's GPU).  Nothing is exchanged while the boxes step;
the only collectives are the max over ranks of the device time and a final
gather of per-box metrics to rank 0.  This replaces the reference's one
process per box (optim/run_tour.py:40-48 launches a janus-sim process per
parameter set): the boxes of a rank share every stage's launch instead.

The partition balances a cost model of a batched step, measured on one B200
with the 64-box ensemble (25.1 M particles, sum of M^3 = 3.8e8 grid cells):
the walks, the interpolation, the sort and half the deposit scale with the
particles (1.14e-6 ms each), the FFTs and the other half of the deposit
with the grid cells (4.8e-8 ms each), so a box costs
n_particles + GRID_WEIGHT * M^3 particle-equivalents.
"""
from __future__ import annotations

GRID_WEIGHT = 0.042


def box_cost(n_particles: int, pm_grid: int) -> float:
    """Particle-equivalent cost of one box in a batched step."""
    return float(n_particles) + GRID_WEIGHT * float(pm_grid) ** 3


def partition(costs, world_size: int):
    """Longest-processing-time-first assignment of boxes to ranks: boxes by
    decreasing cost (ties by index), each to the rank with the least load so
    far (ties to the lowest rank).  Deterministic, so every rank computes the
    same partition without communicating.  Returns, per rank, its box indices
    in increasing order.  The heaviest rank carries at most 4/3 of the
    optimal makespan (Graham's bound)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    costs = [float(c) for c in costs]
    if any(c < 0 for c in costs):
        raise ValueError("costs must be >= 0")
    load = [0.0] * world_size
    share = [[] for _ in range(world_size)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world_size), key=lambda q: (load[q], q))
        share[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in share]


def loads(costs, shares):
    """Summed cost of each rank's share."""
    return [sum(float(costs[i]) for i in s) for s in shares]


def gather(obj, world_size: int):
    """Rank 0 receives every rank's object (a list in rank order), the others
    None; world_size 1 needs no process group.  Every rank must call it, in
    the same order relative to the other collectives."""
    if world_size == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world_size if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
