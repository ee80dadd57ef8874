"""Multi-rank host logic on CPU (gloo, world size 2): disjoint seeds, the
round-robin shard, and the max-over-ranks timing the bench uses."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from oflow import multigpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = multigpu.rank_seeds(rank, world, 4, base=10)
        mine = multigpu.shard(list(range(11)), rank, world)
        t = multigpu.max_over_ranks(1.5 + rank)
        obj = [None] * world
        dist.all_gather_object(obj, seeds)
        q.put((rank, seeds, mine, t, obj))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, m0, t0, all0), (r1, s1, m1, t1, _) = res
    assert s0 == [10, 11, 12, 13] and s1 == [14, 15, 16, 17]
    assert not set(all0[0]) & set(all0[1])
    assert m0 == [0, 2, 4, 6, 8, 10] and m1 == [1, 3, 5, 7, 9]
    assert t0 == t1 == 2.5


def test_single_process_helpers():
    assert multigpu.max_over_ranks(3.0) == 3.0
    assert multigpu.shard([1, 2, 3], 0, 1) == [1, 2, 3]
    with pytest.raises(ValueError):
        multigpu.rank_seeds(2, 2, 4)
