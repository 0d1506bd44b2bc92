"""Data-parallel imaging over several GPUs: one process per GPU, clips sharded.

Partially coherent imaging of independent clips has no exchange step: each
rank images its own clips and only the results travel (the reference images
clips one at a time on one host, expose/aerial_image.py:502-548). The shard
plan balances ranks by cost (pixels x coherent systems, so uneven clip sizes
spread evenly) and is deterministic, so every rank computes the same plan
without communicating. ``gather_results`` reassembles the outputs in input
order with one all-gather of pickled host arrays (gloo or NCCL process
group); device tensors stay on their rank unless gathered.
"""

from __future__ import annotations

from typing import Callable, Sequence


def shard_plan(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assign item indices to `world` ranks, largest first onto the least
    loaded rank (ties to the lower rank); each rank's list is in input order."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def clip_cost(n_pixels: int, n_systems: int = 1) -> float:
    """Relative cost of imaging one clip: its pixels times coherent systems."""
    return float(n_pixels) * float(n_pixels) * float(max(1, n_systems))


def run_sharded(items: Sequence, costs: Sequence[float], fn: Callable[[list], list], rank: int, world: int):
    """Run fn on this rank's share of `items`; returns (indices, results)."""
    mine = shard_plan(costs, world)[rank]
    out = fn([items[i] for i in mine]) if mine else []
    if len(out) != len(mine):
        raise RuntimeError(f"rank {rank}: fn returned {len(out)} results for {len(mine)} items")
    return mine, list(out)


def gather_results(n_items: int, mine: list[int], results: list, group=None) -> list:
    """All-gather every rank's (indices, results) and return the results of
    all items in input order (on every rank)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    box = [None] * world
    dist.all_gather_object(box, (list(mine), list(results)), group=group)
    full: list = [None] * n_items
    seen = 0
    for idx, res in box:
        for i, r in zip(idx, res):
            if full[i] is not None:
                raise RuntimeError(f"item {i} produced by two ranks")
            full[i] = r
            seen += 1
    if seen != n_items:
        raise RuntimeError(f"gathered {seen} of {n_items} results")
    return full


__all__ = ["shard_plan", "clip_cost", "run_sharded", "gather_results"]
