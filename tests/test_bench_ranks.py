"""Replica runs over several ranks (bench.py --gpus N): the whole-job time is
the slowest rank's and the work is the sum over ranks.  Checked with two gloo
ranks on the CPU (the same reduction runs over NCCL on GPUs)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, w = bench.combine_ranks(dist, torch, 1.0 + rank, 100.0 * (rank + 1), "cpu")
        out[rank] = (t, w)
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_sum_work():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        assert out[r] == (2.0, 300.0)
