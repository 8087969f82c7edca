"""Multi-rank placement of independent problems, exercised with two gloo
ranks on CPU: every problem lands on exactly one rank, loads balance, and
the step reduction takes the maximum time and the total converged count."""
import os
import socket

import pytest

from samrai_b200 import parallel


def test_partition_is_disjoint_and_balanced():
    costs = [float(c) for c in range(1, 65)]
    for world in (1, 2, 4, 8):
        parts = parallel.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        assert parallel.imbalance(costs, parts) < 1.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    mine = parallel.shard(costs, rank, world)
    # gather every rank's shard
    t = torch.full((len(costs),), -1, dtype=torch.int64)
    for i in mine:
        t[i] = rank
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, conv = parallel.reduce_step(dist, ms=10.0 * (rank + 1), converged=len(mine))
    q.put((rank, t.tolist(), ms, conv))
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    costs = [3.0, 1.0, 4.0, 1.0, 5.0, 9.0, 2.0, 6.0]
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owners = res[0][1]
    assert res[1][1] == owners
    assert all(o in (0, 1) for o in owners)
    for rank, _, ms, conv in res:
        assert ms == 20.0
        assert conv == len(costs)
