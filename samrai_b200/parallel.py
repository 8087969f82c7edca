"""Multi-GPU placement of independent FAC problems.

The batched workloads are sets of independent hierarchies, so ranks take
disjoint shards and never exchange field data (the reference's MPI
decomposition exchanges ghosts between ranks, tbox/Schedule.C:209-560; with
one hierarchy per problem there is nothing to exchange).  Only scalars cross
ranks: convergence counts and the step time (maximum over ranks).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time partition of problems over `world` ranks:
    each problem goes to the least loaded rank, largest first.  Returns the
    problem indices of every rank, each list in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(v) for v in out]


def shard(costs: Sequence[float], rank: int, world: int) -> List[int]:
    return partition(costs, world)[rank]


def imbalance(costs: Sequence[float], parts: List[List[int]]) -> float:
    """max rank load / mean rank load."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def reduce_step(dist, ms: float, converged: int, device=None):
    """Max step time and total converged problems over ranks (any backend)."""
    import torch
    t = torch.tensor([ms, float(converged)], dtype=torch.float64, device=device)
    m = t.clone()
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    s = t.clone()
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    return float(m[0].item()), int(round(s[1].item()))
