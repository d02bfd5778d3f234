"""Multi-process host logic on CPU (gloo, world size 2): the max-over-ranks
timing reduction and the replicas-only split of independent problems."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank])
        items = bench.replica_items(513, rank, world)
        q.put((rank, got, items))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_split_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(world):
        r, got, items = q.get(timeout=120)
        out[r] = (got, items)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert out[r][0] == [2.0, 10.0]
    assert out[0][1] == (0, 257) and out[1][1] == (257, 513)


def _batch_worker(rank, world, port, q):
    """One replica of the batched leg with a stand-in solver: the rank takes
    its shard of the 512-instance configuration, 'solves' it (every
    instance converges; wall time proportional to the shard's rows) and
    reduces the whole-job throughput exactly as bench.batch_solve_bench."""
    import numpy as np
    import torch.distributed as dist
    import bench
    from amigo_b200.problems.cartpole import batch_config
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = batch_config(k=512, seed=0)
        mine = bench.shard(full.inst, rank, world)
        ids = [full.inst.index(m) for m in mine]
        wall = 1e-6 * sum(m.n for m in mine)
        conv = np.ones(len(mine), bool)
        wall_all, = bench.max_over_ranks([wall])
        conv_all, = bench.sum_over_ranks([int(conv.sum())])
        q.put((rank, ids, wall_all, conv_all))
    finally:
        dist.destroy_process_group()


def test_batch_replicas_split_and_reduce_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_batch_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, ids, wall_all, conv_all = q.get(timeout=180)
        out[r] = (ids, wall_all, conv_all)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ids0, ids1 = out[0][0], out[1][0]
    assert not set(ids0) & set(ids1)                  # disjoint shards
    assert sorted(ids0 + ids1) == list(range(512))    # covering the batch
    assert out[0][2] == out[1][2] == 512              # summed solves
    assert out[0][1] == out[1][1] > 0                 # slowest rank's time


def test_replica_items_cover_all():
    import bench
    for n in (0, 1, 7, 512, 1000):
        for w in (1, 2, 3, 8):
            spans = [bench.replica_items(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for a, b in zip(spans, spans[1:]):
                assert a[1] == b[0]
