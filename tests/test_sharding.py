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


def _failing_worker(rank, world, port, q, mode):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    if mode == "never_joins" and rank == 1:
        return  # the rank dies before it joins the group
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=5))
    except Exception as e:  # rendezvous gave up: the other rank never came
        q.put((rank, "init", type(e).__name__))
        return
    if mode == "raises" and rank == 1:
        dist.destroy_process_group()
        raise SystemExit(3)  # fails between steps, with nothing in flight
    try:
        sharding.max_over_ranks(1.0)  # the next step's collective
        q.put((rank, "ok", ""))
    except Exception as e:
        q.put((rank, "collective", type(e).__name__))


@pytest.mark.parametrize("mode", ["raises", "never_joins"])
def test_rank_failure_is_seen_by_the_other(mode):
    """A rank that fails between steps (or never joins) makes the surviving
    rank's next collective (or the rendezvous) end with an error within the
    group's short timeout instead of hanging."""
    import time
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29400 + os.getpid() % 150 + (50 if mode == "raises" else 0)
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q, mode)) for r in range(2)]
    t0 = time.time()
    for p in procs:
        p.start()
    rank, where, err = q.get(timeout=90)
    for p in procs:
        p.join(timeout=60)
    assert rank == 0 and where in ("init", "collective") and err, (rank, where, err)
    assert time.time() - t0 < 90
    assert procs[1].exitcode != 0 or mode == "never_joins"


def test_no_group_is_identity():
    assert sharding.max_over_ranks(3.0) == 3.0
    assert sharding.whole_job_rate(10, 2.0) == 5.0


def _bench():
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_starts_its_own_ranks(tmp_path, monkeypatch):
    """`bench.py --gpus N` without torchrun re-runs itself under
    torch.distributed.run with N ranks; inside a rank (WORLD_SIZE set) or for
    N = 1 it runs in place.  The command is run here for real on a stand-in
    script whose two ranks meet over gloo."""
    import subprocess
    import sys
    bench = _bench()
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    cmd = bench.launch_command(4, ["--gpus", "4", "--steps", "3"], port=29123)
    assert cmd[:3] == [sys.executable, "-m", "torch.distributed.run"]
    assert "--nproc-per-node=4" in cmd and cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-4:] == ["--gpus", "4", "--steps", "3"] and cmd[-5].endswith("bench.py")
    assert bench.maybe_launch(1, []) is None
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.maybe_launch(2, []) is None
    monkeypatch.delenv("WORLD_SIZE")
    script = tmp_path / "rank.py"
    script.write_text(
        "import os, datetime, torch, torch.distributed as dist\n"
        "dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=60))\n"
        "t = torch.tensor([float(os.environ['RANK']) + 1])\n"
        "dist.all_reduce(t)\n"
        "os.write(1, f\"sum={int(t.item())}:{os.environ['WORLD_SIZE']}\\n\".encode())\n"
        "dist.destroy_process_group()\n")
    out = subprocess.run(bench.launch_command(2, [], port=29000 + os.getpid() % 500,
                                              script=str(script)),
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.count("sum=3:2") == 2, out.stdout
