"""Multi-GPU batch sharding, host logic on CPU: gloo, world size 2."""
import os

import pytest
import torch.multiprocessing as mp

from ffta_b200 import sharding


@pytest.mark.parametrize("total,world", [(16384, 2), (16384, 8), (7, 3), (0, 2), (5, 8)])
def test_shard_ranges_partition(total, world):
    seen = []
    for r in range(world):
        s, c = sharding.shard_range(total, world, r)
        seen.extend(range(s, s + c))
    assert seen == list(range(total))
    sizes = [sharding.shard_range(total, world, r)[1] for r in range(world)]
    assert max(sizes) - min(sizes) <= 1


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        start, count = sharding.shard_range(10, world, rank)
        # each rank "times" its shard; rank 1 is the slow one
        local = 0.5 + rank
        mx = sharding.max_over_ranks(local)
        rate = sharding.whole_job_rate(count, local)
        got = torch.zeros(10)
        got[start:start + count] = 1
        dist.all_reduce(got)
        q.put((rank, mx, rate, got.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 200
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rate, got in res:
        assert mx == 1.5  # the slower rank's time
        assert rate == pytest.approx(10 / 1.5)  # all units over the max time
        assert got == [1.0] * 10  # every column owned by exactly one rank


def test_no_group_is_identity():
    assert sharding.max_over_ranks(3.0) == 3.0
    assert sharding.whole_job_rate(10, 2.0) == 5.0
