"""Multi-rank sharding of a sweep, on CPU with the gloo backend (world 2).

The data path has no collective: rank r sweeps rows r, r + stride, ... of
every class.  This checks, with real torch.distributed ranks, that the
shards are disjoint, that their union is the rows r < world (mod stride),
that each rank's shard matches the one-rank sample in size (weak scaling),
and that the job-level reductions give the summed work and the slowest
rank's time.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from simint_b200.shard import shard_rows, check_world, reduce_count_sum, reduce_time_max  # noqa: E402

NROWS = [1, 7, 40, 123, 1000]
STRIDE = 5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        check_world(world, STRIDE)
        mine = [shard_rows(n, STRIDE, rank) for n in NROWS]
        allr = [None] * world
        dist.all_gather_object(allr, mine)
        work = sum(len(r) for r in mine)
        total = reduce_count_sum(dist, work)
        slow = reduce_time_max(dist, 10.0 + rank)
        if rank == 0:
            q.put((allr, total, slow))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_are_disjoint_and_reduce():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    allr, total, slow = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for k, n in enumerate(NROWS):
        a, b = set(allr[0][k]), set(allr[1][k])
        assert not (a & b)
        assert a | b == {r for r in range(n) if r % STRIDE < world}
        # weak scaling: each rank's shard is the one-rank sample's size (within one row)
        assert abs(len(allr[1][k]) - len(shard_rows(n, STRIDE, 0))) <= 1
    assert total == sum(len(allr[r][k]) for r in range(world) for k in range(len(NROWS)))
    assert slow == 11.0


def test_world_larger_than_stride_is_refused():
    with pytest.raises(ValueError):
        check_world(6, 5)
    assert shard_rows(10, 5, 7) == shard_rows(10, 5, 2)
