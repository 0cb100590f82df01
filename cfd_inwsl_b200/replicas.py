"""Replicas over GPUs for the work that has no exchange step: the batched
configuration's independent cases, and independent adjoint solves.

One process per GPU (torch.distributed). Every rank computes the same
assignment of cases from their costs without communicating, runs its share on
its own GPU (a BlockBatch of its cases), and the results are gathered on rank
0 at the end: the gather is the only collective, none is on the data path.

The cost of a 2D case of N x N cells run to a fixed time is N^2 cells times a
CFL step count that grows as N, so N^3 (N^(dim+1) in general); cases are
assigned by the longest-processing-time rule (largest first, each to the rank
with the least cost so far), whose largest share is at most 4/3 of the best
possible.
"""
from __future__ import annotations

from typing import Callable, Sequence


def case_cost(n: int, dim: int = 2) -> float:
    """Relative cost of a case of n cells per side run to a fixed time."""
    return float(n) ** (dim + 1)


def partition_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the cases of each rank (each list ascending). Largest cost
    first (ties by index), each to the rank with the smallest total so far
    (ties: the lowest rank), so every rank derives the same partition."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    share: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        share[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in share]


def share_loads(costs: Sequence[float], shares: Sequence[Sequence[int]]) -> list[float]:
    return [sum(float(costs[i]) for i in s) for s in shares]


def run_sharded(items: Sequence, run_share: Callable[[list[int]], list], costs: Sequence[float], rank: int,
                world: int, group=None):
    """Run this rank's share of `items` and gather every result on rank 0.

    run_share(indices) returns the results of those items in that order.
    Returns the results of all items in their original order on rank 0 and
    None on the other ranks; with world == 1 it just runs everything."""
    shares = partition_by_cost(costs, world)
    mine = shares[rank]
    out = run_share(mine)
    if len(out) != len(mine):
        raise RuntimeError(f"rank {rank}: {len(out)} results for {len(mine)} cases")
    if world == 1:
        return list(out)
    import torch.distributed as dist
    got = [None] * world if rank == 0 else None
    dist.gather_object((mine, list(out)), got, dst=0, group=group)
    if rank != 0:
        return None
    res = [None] * len(items)
    for idx, vals in got:
        for i, v in zip(idx, vals):
            res[i] = v
    return res
