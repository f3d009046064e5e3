"""The multi-GPU path of bench.py (replicas, no collective on the data path): the job's time is the
slowest rank's (all_reduce MAX, then a barrier) and the rate counts every rank's units. Run as two
gloo ranks on the CPU, as the GPU ranks run over NCCL."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, torch.device("cpu"))
        dist.barrier()
        out[rank] = ms
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_slowest_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == 15.0


def test_rate_counts_every_rank():
    assert bench.whole_job_rate(16_000_000, 1, 1000.0) == pytest.approx(16.0)
    assert bench.whole_job_rate(16_000_000, 8, 1000.0) == pytest.approx(128.0)
    assert bench.max_over_ranks(3.0, None, None) == 3.0
