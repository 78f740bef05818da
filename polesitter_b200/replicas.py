"""Multi-GPU runs of the FMM tick: independent replicas, one process per GPU.

One system's tick has no exchange step (north star: one GPU per system), so
`bench.py --gpus N` runs N independent replicas and only needs two
collectives on the host side: a barrier around the timed region and the
maximum of the per-rank elapsed times (the job is as slow as its slowest
rank).  Works on any torch.distributed backend (NCCL on the GPUs, gloo in the
CPU tests)."""

from __future__ import annotations


def job_time(local_seconds: float, device=None) -> float:
    """Max over ranks of ``local_seconds`` (the local value if not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_seconds)
    t = torch.tensor([float(local_seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: int, local_seconds: float, device=None) -> float:
    """Units processed by all ranks per second of the slowest rank (weak scaling)."""
    import torch.distributed as dist
    world = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    return world * units_per_rank / job_time(local_seconds, device)
