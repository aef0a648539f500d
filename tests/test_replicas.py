"""Multi-GPU runs are replicas: every rank solves the whole workload, the step
time is the slowest rank's (max over ranks) and the throughput the sum over
ranks.  The host logic of that path runs here as two gloo ranks on the CPU;
the reference arm under torchrun runs on rank 0 only."""
import os
import socket
import subprocess
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sys.path.insert(0, REPO)
        import bench
        ms = [120.0, 150.0][rank]          # rank 1 is the slower one
        slow = bench.max_over_ranks(ms, world, "cpu")
        out[rank] = (slow, bench.replica_throughput(world, 64, slow))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_step_and_the_summed_throughput():
    world = 2
    out = mp.get_context("spawn").Manager().dict()   # no fork of a threaded process
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1]
    slow, value = out[0]
    assert slow == 150.0
    assert abs(value - 2 * 64 / 0.150) < 1e-9


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert abs(bench.replica_throughput(1, 64, 1000.0) - 64.0) < 1e-12


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun, ranks other than 0 of `bench.py --impl reference` exit 0
    without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
