"""Multi-GPU mode of bench.py: independent replicas, one per rank, timed as
the slowest rank. The host logic runs here as two gloo ranks on CPU: the max
over ranks, the whole-job rate, per-rank seeds, and the reference arm's rank-0
rule. No GPU, no data-path collective (the replicas never exchange fields)."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r "took" 10 + r seconds for 100 steps: the job is timed by the slowest
        t = bench.reduce_max(10.0 + rank, dist, "cpu")
        rate = bench.aggregate_rate(100, t, world)
        # each rank relaxes its own seeded replica
        f = bench.workload(64, rank)[3]
        digest = float(np.abs(f).sum())
        gathered = [None] * world
        dist.all_gather_object(gathered, digest)
        out[rank] = (t, rate, gathered)
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_seeds():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, start_method="spawn", join=True)
    for rank in range(world):
        t, rate, digests = out[rank]
        assert t == 11.0
        assert rate == pytest.approx(100 * world / 11.0)
        assert digests[0] != digests[1]


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    args = argparse.Namespace(size=64, steps=2, cpu_steps=2, reps=1)
    bench.run_reference(args, rank=1, world=2)
    assert capsys.readouterr().out == ""
