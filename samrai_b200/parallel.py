"""Multi-GPU placement of FAC problems and of one hierarchy's patches.

Batched workloads (config 5) are sets of independent hierarchies: ranks take
disjoint, cell-balanced shards (`partition`) and exchange no field data, only
scalars (convergence counts, the step time as the maximum over ranks).

One large hierarchy (config 2 style) is split by patches, as the reference's
MPI decomposition does: each level's patches go to ranks in Morton order of
their box centres with cell-balanced cuts (`morton_partition`, the
space-filling-curve split of SAMRAI's CascadePartitioner and
TreeLoadBalancer), and each ghost fill's element table (`fac_fill_table`,
the transactions of the reference's RefineSchedule) is split into local
copies and per-peer send and receive lists (`FillPlan`), as
tbox::Schedule splits transactions into local, send and receive sets
(tbox/Schedule.C:98-175) before it communicates (:209-560).  `exchange`
moves the remote values with point-to-point messages of packed buffers
(torch.distributed: NCCL between GPUs, gloo on CPU) into the destination's
ghost cells; every source element is an interior cell and every destination
a ghost cell, so one exchange completes a fill.
"""
from __future__ import annotations

import heapq
from typing import Dict, List, Sequence

import numpy as np


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


# ---------------------------------------------------------------------------
# one hierarchy over ranks
# ---------------------------------------------------------------------------

def _morton_key(x, y, z, bits=21):
    k = 0
    for b in range(bits):
        k |= ((x >> b) & 1) << (3 * b) | ((y >> b) & 1) << (3 * b + 1) | ((z >> b) & 1) << (3 * b + 2)
    return k


def morton_partition(boxes: np.ndarray, world: int) -> np.ndarray:
    """Owner rank of each patch of one level: patches sorted by the Morton
    code of their box centres (lo + hi, so integers), then cut into `world`
    contiguous runs of about equal cell counts."""
    b = np.asarray(boxes, dtype=np.int64).reshape(-1, 6)
    cells = np.prod(b[:, 3:] - b[:, :3] + 1, axis=1)
    c = b[:, :3] + b[:, 3:]
    c = c - c.min(axis=0)
    keys = [_morton_key(int(x), int(y), int(z)) for x, y, z in c]
    order = sorted(range(len(b)), key=lambda i: (keys[i], i))
    owner = np.zeros(len(b), dtype=np.int64)
    total = float(cells.sum())
    acc = 0.0
    for i in order:
        # the rank whose share the middle of this patch falls in
        mid = acc + 0.5 * cells[i]
        owner[i] = min(world - 1, int(mid * world / total))
        acc += cells[i]
    return owner


def element_owner(prob, ln: int, patch_owner: np.ndarray) -> np.ndarray:
    """Owner rank of every element of a level's ghost-1 cell array."""
    from . import configs
    sizes = [int(np.prod(configs.cell_shape(prob.dim, b, 1)[1])) for b in prob.levels[ln].boxes]
    return np.repeat(np.asarray(patch_owner, dtype=np.int64), sizes)


class FillPlan:
    """One rank's part of a ghost fill: the copies whose source and
    destination it owns, and per peer the elements it sends (sources it owns
    whose destination the peer owns) and receives, both sides listed in the
    order of the global table, so the packed buffers match."""

    def __init__(self, dst, src, dst_owner, same_owner, coarse_owner, rank: int):
        dst = np.asarray(dst, dtype=np.int64)
        src = np.asarray(src, dtype=np.int64)
        coarse = src < 0
        sidx = np.where(coarse, -src - 1, src)
        sown = np.empty(len(src), dtype=np.int64)
        sown[~coarse] = same_owner[sidx[~coarse]]
        if coarse.any():
            if coarse_owner is None:
                raise ValueError("the table has coarse-level sources: give their owners")
            sown[coarse] = coarse_owner[sidx[coarse]]
        downer = dst_owner[dst]
        self.rank = rank
        mine = downer == rank
        loc = mine & (sown == rank)
        self.local_dst, self.local_src, self.local_coarse = dst[loc], sidx[loc], coarse[loc]
        self.recv: Dict[int, tuple] = {}
        self.send: Dict[int, tuple] = {}
        for q in np.unique(np.concatenate([sown[mine], downer[sown == rank]])):
            q = int(q)
            if q == rank:
                continue
            r = mine & (sown == q)
            if r.any():
                self.recv[q] = (dst[r],)
            t = (downer == q) & (sown == rank)
            if t.any():
                self.send[q] = (sidx[t], coarse[t])

    def volume(self):
        """(local copies, elements sent, elements received)"""
        return (len(self.local_dst), sum(len(v[0]) for v in self.send.values()),
                sum(len(v[0]) for v in self.recv.values()))


def exchange(plan: FillPlan, x, x_coarse, dist):
    """Run one rank's part of a fill on torch tensors: x is the level's
    ghost-1 array, x_coarse the coarser level's (or None).  Sends are packed
    from interior cells, received values unpacked into ghost cells; the
    messages go to every peer in rank order (so two ranks never both wait on
    a receive first)."""
    import torch
    dev = x.device

    def take(idx, coarse):
        idx_t = torch.as_tensor(idx, device=dev)
        if coarse is None or not np.any(coarse):
            return x.index_select(0, idx_t)
        c_t = torch.as_tensor(coarse, device=dev)
        out = x.index_select(0, torch.where(c_t, torch.zeros_like(idx_t), idx_t))
        return torch.where(c_t, x_coarse.index_select(0, torch.where(c_t, idx_t,
                                                                        torch.zeros_like(idx_t))),
                           out)

    reqs, bufs = [], {}
    for q in sorted(set(plan.send) | set(plan.recv)):
        if q in plan.send:
            sb = take(*plan.send[q]).contiguous()
            reqs.append(dist.isend(sb, dst=q))
            bufs[("s", q)] = sb
        if q in plan.recv:
            rb = torch.empty(len(plan.recv[q][0]), dtype=x.dtype, device=dev)
            reqs.append(dist.irecv(rb, src=q))
            bufs[("r", q)] = rb
    if len(plan.local_dst):
        vals = take(plan.local_src, plan.local_coarse)
        x.index_copy_(0, torch.as_tensor(plan.local_dst, device=dev), vals)
    for r in reqs:
        r.wait()
    for q in plan.recv:
        x.index_copy_(0, torch.as_tensor(plan.recv[q][0], device=dev), bufs[("r", q)])
