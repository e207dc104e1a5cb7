"""CPU, two processes over gloo: the multi-rank host logic.  The replica
timing of bench.py (each rank runs its own copy of the workload, the step
time is the slowest rank's, the job's rate counts every rank's particles),
and the target shares of pepc_b200.shard_range (contiguous, disjoint,
covering, 64-aligned), gathered across the ranks."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
import pepc_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def _share_worker(rank, world, port, n, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t0, t1 = pepc_b200.shard_range(n, rank, world)
        mine = torch.tensor([t0, t1], dtype=torch.int64)
        every = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(every, mine)
        out[rank] = [tuple(int(v) for v in e) for e in every]
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [10007, 64, 5])
def test_target_shares_cover_the_particles(n):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_share_worker, args=(world, _free_port(), n, out), nprocs=world,
                       join=True, start_method="spawn")
    shares = out[0]
    assert out[1] == shares
    assert shares[0][0] == 0 and shares[-1][1] == n
    for (a0, a1), (b0, b1) in zip(shares, shares[1:]):
        assert a1 == b0 and a0 <= a1
    assert all(t0 % 32 == 0 for t0, _ in shares)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(7.0, None, torch.device("cpu")) == 7.0


def _gather_worker(rank, world, port, n, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t0, t1 = pepc_b200.shard_range(n, rank, world)
        # the "fields" of a share: field f of target t is 10 f + t
        local = torch.stack([10.0 * f + torch.arange(t0, t1, dtype=torch.float64)
                             for f in range(5)])
        full = pepc_b200.gather_shards(local, n, rank, world)
        out[rank] = full.numpy().tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [1000, 4096, 33])
def test_gather_shards_rebuilds_the_fields(n):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_gather_worker, args=(world, _free_port(), n, out), nprocs=world,
                       join=True, start_method="spawn")
    want = [[10.0 * f + t for t in range(n)] for f in range(5)]
    assert out[0] == want and out[1] == want


def test_bench_refuses_a_rank_count_that_differs_from_gpus():
    # --gpus N must be the number of ranks the launcher started
    import subprocess
    import sys
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "--gpus 2" in r.stderr
