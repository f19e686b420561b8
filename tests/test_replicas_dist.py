"""Replicas across ranks: sharding and the job-wide rate, with two gloo ranks on CPU."""
import os
import socket

import pytest

from qcd_2d_gpu_b200.replicas import job_rate, shard


def test_shard_covers_every_replica_once():
    items = list(range(97))
    parts = [shard(items, r, 4) for r in range(4)]
    assert sorted(sum(parts, [])) == items
    assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        shard(items, 4, 4)


def test_job_rate_single_process():
    rate, ms = job_rate(1000.0, 2.0)
    assert rate == 500000.0 and ms == 2.0


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r processes its shard of 10 replicas in (r + 1) ms
        mine = shard(range(10), rank, world)
        rate, ms = job_rate(float(len(mine)), float(rank + 1), dist)
        out[rank] = (rate, ms)
    finally:
        dist.destroy_process_group()


def test_job_rate_two_gloo_ranks():
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()  # no fork: the parent may hold CUDA state
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    # 10 replicas in total, the slowest rank took 2 ms
    assert out[0] == out[1] == (10 / 2e-3, 2.0)
