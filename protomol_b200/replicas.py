"""Replicas across GPUs: one process per GPU, independent systems, no
collective on the data path.

A single system of the sizes served here does not shard (that would need
spatial decomposition with a halo exchange every step and a PME all-to-all).
What spreads over several GPUs is whole systems: the requests of a stream or
the boxes of an ensemble are partitioned across the ranks, every rank runs
its share on its own device, and the only collectives are the host-side
bookkeeping below (the max-over-ranks time and the gathered summaries).
"""
from __future__ import annotations

import heapq


def partition(costs: list[float], world: int) -> list[list[int]]:
    """Deterministic longest-processing-time assignment of items (by
    estimated cost) to `world` ranks: every item goes to exactly one rank
    and the largest per-rank total stays within 4/3 of the optimum."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + costs[k], r))
    for lst in out:
        lst.sort()
    return out


def request_cost(req) -> float:
    """Relative device time of a served request: atoms x steps (an energy
    evaluation counts as one step), plus a fixed set-up share."""
    steps = req.steps if req.kind == "segment" else 1
    return req.n_atoms * max(1, steps) + 2.0e5


def my_share(items: list, world: int, rank: int, cost=request_cost) -> list:
    """The items rank `rank` of `world` runs."""
    parts = partition([cost(x) for x in items], world)
    return [items[k] for k in parts[rank]]


def max_over_ranks(value: float, dist=None) -> float:
    """The largest value over all ranks (the job's time is its slowest
    rank's); `dist` is torch.distributed with an initialised group, or None
    for a single process."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_summaries(summary: dict, dist=None) -> list[dict]:
    """Every rank's summary dictionary, in rank order, on every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [summary]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, summary)
    return out
