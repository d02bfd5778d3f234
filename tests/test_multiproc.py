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


def test_replica_items_cover_all():
    import bench
    for n in (0, 1, 7, 512, 1000):
        for w in (1, 2, 3, 8):
            spans = [bench.replica_items(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for a, b in zip(spans, spans[1:]):
                assert a[1] == b[0]
