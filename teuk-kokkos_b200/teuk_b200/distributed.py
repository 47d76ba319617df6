"""Rank plumbing for multi-GPU runs of the engine.

One process per GPU.  The path does not shard inside a solve (every RK stage
chains SBP derivatives across a 16-point closure), so ranks own disjoint sets
of independent solves and the data path has no collective.  The collectives
here are the barrier that brackets a timed region and the reductions of its
per-rank results (max of device time, sum of work), on NCCL for GPU ranks
and gloo for CPU tests.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass(frozen=True)
class RankInfo:
    rank: int
    world_size: int
    local_rank: int


def rank_info() -> RankInfo:
    """RANK / WORLD_SIZE / LOCAL_RANK of a torchrun launch (0 / 1 / 0 alone)."""
    return RankInfo(int(os.environ.get("RANK", "0")),
                    int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_seconds: float = 120.0, device=None) -> RankInfo:
    """Join the process group when WORLD_SIZE > 1 (rendezvous on
    127.0.0.1 unless MASTER_ADDR says otherwise)."""
    import torch.distributed as dist

    info = rank_info()
    if info.world_size > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        kwargs = {"timeout": timedelta(seconds=timeout_seconds)}
        if device is not None:
            kwargs["device_id"] = device
        dist.init_process_group(backend, **kwargs)
    return info


def shard(count: int, rank: int, world_size: int) -> range:
    """Balanced contiguous block of the solve indices owned by `rank`."""
    if count < 0 or world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("invalid shard request")
    begin = count * rank // world_size
    end = count * (rank + 1) // world_size
    return range(begin, end)


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.barrier()


def _reduce(value: float, op, device) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, device="cpu") -> float:
    import torch.distributed as dist

    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value: float, device="cpu") -> float:
    import torch.distributed as dist

    return _reduce(value, dist.ReduceOp.SUM, device)


def whole_job_rate(local_units: float, local_seconds: float,
                   device="cpu") -> tuple[float, float]:
    """(units of all ranks / slowest rank's time, slowest time): the
    whole-job throughput of a timed region that every rank ran."""
    total = sum_over_ranks(local_units, device)
    slowest = max_over_ranks(local_seconds, device)
    return total / slowest, slowest


def finalize() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.destroy_process_group()
