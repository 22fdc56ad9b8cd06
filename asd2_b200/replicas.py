"""Replica bookkeeping of multi-GPU runs.  The droplet step does not shard
(one pressure system per droplet), so N processes run N independent replicas;
the job's time is the slowest rank's and its throughput counts the units of
every rank.  Host-side only: the same functions run over NCCL (bench.py on
GPUs) and over gloo (the CPU tests)."""
from __future__ import annotations

import datetime
import os


def rank_env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_group(backend: str, timeout_s: float = 120.0):
    """The default process group with a short timeout (ranks that wait on a
    missing peer end with an error instead of hanging); None for one rank."""
    rank, world, _ = rank_env()
    if world <= 1:
        return None
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def job_time(local_seconds: float, dist=None, device: str = "cpu") -> float:
    """The whole job's time: the maximum of the ranks' timed-region seconds."""
    if dist is None:
        return float(local_seconds)
    import torch
    t = torch.tensor([float(local_seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, job_seconds: float) -> float:
    """Units per second of the whole job (every rank's units over the slowest rank's time)."""
    return world * units_per_rank / job_seconds


def reference_rank_runs(rank: int) -> bool:
    """The CPU reference arm runs on rank 0 only; other ranks exit without work."""
    return rank == 0
