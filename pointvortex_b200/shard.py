"""Ensembles across GPUs: one engine per GPU, no data exchange between them.

A batched ensemble (or a serving stream) is split into independent simulations, so several GPUs
run it as replicas of the batch engine. Each rank takes a share of the simulations and runs them
in its own arena; only the final per-simulation results travel, once, to rank 0. The partition
is the longest-processing-time rule on the estimated cost of each simulation (N^2 times the
measured relative pair cost of its geometry), which balances the ranks to within one simulation.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

from .serve import PAIR_COST


def simulation_cost(geometry: str, n: int) -> float:
    """Estimated cost of one velocity evaluation, in plane-pair units."""
    return PAIR_COST[geometry] * float(n) * float(n)


def partition(costs: Sequence[float], world: int) -> list[int]:
    """Rank of each simulation: the costliest first, each to the least-loaded rank (ties to the
    lower rank). Deterministic, so every rank computes the same assignment on its own."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [(0.0, r) for r in range(world)]
    heapq.heapify(loads)
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(loads)
        owner[i] = r
        heapq.heappush(loads, (load + costs[i], r))
    return owner


def run_sharded(specs: Sequence, cost_of: Callable, run_local: Callable, rank: int, world: int,
                gather: Callable | None = None) -> list | None:
    """Runs this rank's share of `specs` with run_local(list of (index, spec)) -> list of
    (index, result), then gathers every rank's results on rank 0 in spec order.
    gather(obj) -> list of every rank's obj (torch.distributed.all_gather_object under a process
    group); without one (a single process) the local results are returned."""
    owner = partition([cost_of(s) for s in specs], world)
    mine = [(i, s) for i, s in enumerate(specs) if owner[i] == rank]
    local = run_local(mine)
    parts = gather(local) if gather is not None else [local]
    if rank != 0:
        return None
    merged = [None] * len(specs)
    for part in parts:
        for i, result in part:
            merged[i] = result
    return merged


def torch_gather(obj) -> list:
    """all_gather_object over the default process group (gloo or NCCL)."""
    import torch.distributed as dist
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
