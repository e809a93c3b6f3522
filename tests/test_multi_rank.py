"""The bench's multi-rank plumbing on CPU: two gloo ranks, replicas timed as the slowest rank.

Each GPU of a run steps its own replica of the workload (no data-path collective);
the job's time is the maximum of the ranks' times and its throughput counts every
rank's bodies. This checks that reduction and arithmetic with torch.distributed over
gloo (world size 2, rendezvous on 127.0.0.1), as bench.py uses them under torchrun.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slower replica
        job_ms = bench.max_over_ranks(dist, local_ms, device="cpu")
        value = bench.replica_throughput(1000, 10, world, job_ms / 1000.0)
        q.put((rank, job_ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_count_all_bodies():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, job_ms, value in out:
        assert job_ms == pytest.approx(150.0)
        assert value == pytest.approx(1000 * 10 * 2 / 0.150)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, 12.5) == 12.5
    assert bench.replica_throughput(131072, 60, 1, 0.3) == pytest.approx(131072 * 60 / 0.3)


def test_clock_sampler_gpu_id(monkeypatch):
    """The rank's nvidia-smi id: its CUDA_VISIBLE_DEVICES entry when nvidia-smi knows it,
    else the local rank (unset variable, or nvidia-smi missing or not knowing the entry)."""
    import subprocess

    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.delenv("CUDA_VISIBLE_DEVICES", raising=False)
    assert bench.smi_gpu_id(3) == "3"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "4,5,6,7")

    def known(cmd, **kw):
        return subprocess.CompletedProcess(cmd, 0, stdout="5\n", stderr="")

    monkeypatch.setattr(bench.subprocess, "run", known)
    assert bench.smi_gpu_id(1) == "5"

    def unknown(cmd, **kw):
        return subprocess.CompletedProcess(cmd, 6, stdout="", stderr="No devices were found")

    monkeypatch.setattr(bench.subprocess, "run", unknown)
    assert bench.smi_gpu_id(1) == "1"

    def missing(cmd, **kw):
        raise FileNotFoundError("nvidia-smi")

    monkeypatch.setattr(bench.subprocess, "run", missing)
    assert bench.smi_gpu_id(2) == "2"
