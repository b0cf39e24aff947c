"""The multi-rank arithmetic of bench.py on CPU: world_size-2 gloo ranks take the
maximum of their times at the same point, and the whole-job rate counts every
rank's units over that maximum (replicas, weak scaling)."""

import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, REPO)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = [12.5, 20.0]  # rank 1 is the slow one
        ms = bench.max_over_ranks(times[rank], dist, "cpu")
        rate = bench.job_rate(1000.0, world, ms)
        dist.barrier()
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_time_and_the_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 20.0
        assert rate == pytest.approx(1000.0 * 2 / 0.020)


def test_single_process_needs_no_collective():
    sys.path.insert(0, REPO)
    import bench

    assert bench.max_over_ranks(7.0, None, "cpu") == 7.0
    assert bench.job_rate(500.0, 1, 10.0) == pytest.approx(50000.0)


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, REPO)
    import bench

    class A:
        steps, warmup = 1, 3

    assert bench.run_reference(A(), rank=1) is None
