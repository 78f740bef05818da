"""Host logic of the multi-GPU (independent replicas) path, on CPU with gloo,
world size 2: the job time is the slowest rank's, throughput counts all ranks."""

from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from polesitter_b200.replicas import job_throughput, job_time
        local = 1.0 + rank  # rank 1 is the slow one
        dist.barrier()
        out[rank] = (job_time(local), job_throughput(10, local))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_weak_scaling_throughput():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        t, thr = out[r]
        assert t == 2.0              # slowest rank
        assert thr == 2 * 10 / 2.0   # all ranks' units over the slowest time


def test_single_process_is_local_value():
    from polesitter_b200.replicas import job_throughput, job_time
    assert job_time(1.5) == 1.5
    assert job_throughput(3, 1.5) == 2.0
