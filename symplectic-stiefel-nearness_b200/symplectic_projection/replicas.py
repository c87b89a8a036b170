"""Several GPUs: independent replicas, one process per GPU.

Instances of the problem are independent (each target is solved on its own), so
a batch spreads over ranks with no data-path collective: every rank solves its
own share with the single-GPU pipeline.  ``partition_by_cost`` splits a list of
target shapes over ranks by estimated cost (largest first onto the least-loaded
rank), and ``max_over_ranks`` / ``gather_results`` are the only collectives,
used for timing and for bringing per-rank results back together.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def target_cost(n: int, k: int, newton_steps: int = 8) -> float:
    """Estimated device time of one target: the tall-skinny products (16 n m^2) plus
    the Newton phase (about 24 products of 2 m^3 per step), m = 2k."""
    m = 2 * k
    return 16.0 * n * m * m + newton_steps * 48.0 * m ** 3


def partition_by_cost(shapes, world: int):
    """Per rank, the indices of the targets it solves: greedy largest-first onto the
    least-loaded rank (ties to the lowest rank), so every rank computes the same plan."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(shapes)), key=lambda i: (-target_cost(*shapes[i]), i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += target_cost(*shapes[i])
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (the step time of a multi-rank run); the value
    itself with no process group."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def gather_results(local: dict, parts):
    """Every rank's {index: result} merged into one list in target order (on every rank)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        merged = dict(local)
    else:
        bucket = [None] * dist.get_world_size()
        dist.all_gather_object(bucket, local)
        merged = {}
        for part in bucket:
            merged.update(part)
    total = sum(len(p) for p in parts)
    if sorted(merged) != list(range(total)):
        raise RuntimeError("results missing or duplicated across ranks")
    return [merged[i] for i in range(total)]
