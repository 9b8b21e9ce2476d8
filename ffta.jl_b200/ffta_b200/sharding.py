"""Batch sharding across GPUs (one process per GPU).

The batched path of FFTA (`_mul_loop!`, src/plan.jl:194-207) transforms
independent columns, so N GPUs split the columns into contiguous blocks and
transform them with no exchange at all.  Only the timing needs the ranks to
meet: a barrier before and after the timed region and the maximum of the
per-rank times (`max_over_ranks`), which is what whole-job throughput is
computed from.  Any torch.distributed backend works (NCCL on GPUs, gloo in
the CPU tests).
"""
from __future__ import annotations


def shard_range(total: int, world: int, rank: int):
    """Contiguous block of `total` columns owned by `rank`: (start, count).

    The first total % world ranks get one extra column, so the blocks cover
    0..total-1 exactly once and differ in size by at most one.
    """
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    if total < 0:
        raise ValueError("negative total")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, seconds_local: float, device=None) -> float:
    """Units per second of the whole job: all ranks' units over the slowest rank's time."""
    import torch
    import torch.distributed as dist
    units = float(units_per_rank)
    if dist.is_available() and dist.is_initialized():
        t = torch.tensor([units], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        units = float(t.item())
    return units / max_over_ranks(seconds_local, device)
