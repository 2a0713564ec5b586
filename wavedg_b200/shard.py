"""Sharding independent WaveHoltz solves across GPUs (one process per GPU).

Batched WaveHoltz problems are independent, so a multi-GPU run splits the problem list
across ranks and each rank runs its share as its own batch: no collective touches the
data path.  The only exchange is the per-problem result record (iterations, residual,
status) gathered at the end, small enough for any backend (gloo on CPU in the tests,
NCCL on the GPUs).

The split balances estimated work: a problem costs about ndof x (RK4 steps per period)
per iteration, the same for every problem's iteration count to first order, so a
longest-processing-time greedy assignment on that cost keeps the ranks within one
problem's cost of each other.
"""
from __future__ import annotations

import math


def cost(ndof: int, n_colloc: int, n_el_side: int, omega: float) -> float:
    """Work of one WaveHoltz iteration: DOF x steps per period, with the period's step count
    from WaveHoltz::WaveHoltz (T = 2 pi / omega, dt = 0.5 h / n^2, h = 2 / n_el_side)."""
    T = 2.0 * math.pi / omega
    dt = 0.5 * (2.0 / n_el_side) / (n_colloc * n_colloc)
    return float(ndof) * math.ceil(T / dt)


def assign(costs, world: int):
    """Problem indices per rank: largest cost first to the least-loaded rank (ties to the lower
    rank), each rank's list in ascending index order.  Deterministic, so every rank computes
    the same split without communicating."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def gather_records(records: dict, world: int):
    """All ranks' {problem index: record} merged on every rank (torch.distributed object
    all-gather; records are small Python values)."""
    import torch.distributed as dist

    if world == 1:
        return dict(records)
    out = [None] * world
    dist.all_gather_object(out, records)
    merged = {}
    for part in out:
        merged.update(part)
    return merged
