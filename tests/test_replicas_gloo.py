"""CPU, two processes over gloo: the replica timing of bench.py -- each rank
runs its own copy of the workload, the step time is the slowest rank's, and
the job's rate counts every rank's particles."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        m = bench.max_over_ranks(ms, dist, torch.device("cpu"))
        out[rank] = (m, bench.job_rate(1000, world, m))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    assert out[0] == out[1]
    m, rate = out[0]
    assert m == 15.0
    assert rate == pytest.approx(1000 * 2 / 15e-3)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(7.0, None, torch.device("cpu")) == 7.0
