"""The multi-GPU form of the bench is replicas: every rank inserts its own
particles, and the job's time is the slowest rank's. This checks that
aggregation (bench.replica_rate) with two gloo ranks on the CPU."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank: int, world: int, port: int, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # Rank r's timed region took 100 + 50 r ms over 4 steps of 1,000 particles.
        ms, rate = bench.replica_rate(100.0 + 50.0 * rank, 4, 1000, dist, torch.device("cpu"))
        results[rank] = (ms, rate)
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    manager = mp.Manager()
    results = manager.dict()
    mp.spawn(rank_main, args=(world, free_port(), results), nprocs=world, join=True)
    slowest = 150.0 / 4
    for rank in range(world):
        ms, rate = results[rank]
        assert ms == pytest.approx(slowest)
        assert rate == pytest.approx(world * 1000 / (slowest / 1e3))


def test_one_rank_without_a_process_group():
    ms, rate = bench.replica_rate(80.0, 4, 1000)
    assert ms == 20.0 and rate == pytest.approx(1000 / 0.02)
