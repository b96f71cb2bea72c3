"""bench.py's multi-GPU form is replicas only: each rank runs the whole path on its own
dataset, the ranks meet at a barrier around the timed steps, and the step time is the
largest over the ranks. These tests run that host logic (the same functions bench.py
calls) as two gloo ranks on the CPU, and check that the reference arm does its work on
rank 0 alone."""

from __future__ import annotations

import datetime
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.replica_barrier(dist, cuda=False)
        step_ms = [120.0, 180.0][rank]  # rank 1 is the slow one
        ms = bench.replica_max(dist, step_ms, device="cpu")
        value = bench.whole_job(world, 1_000_000, ms)
        bench.replica_barrier(dist, cuda=False)
        out.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_the_slowest_rank_and_count_every_ranks_cells():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=10) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 180.0  # every rank reports the slowest rank's time
        assert value == pytest.approx(2 * 1_000_000 / 0.180)


def test_one_rank_is_its_own_maximum():
    import bench

    assert bench.replica_max(None, 42.5, device="cpu") == 42.5
    assert bench.whole_job(1, 1_000_000, 250.0) == pytest.approx(4_000_000.0)


def test_reference_arm_runs_on_rank_zero_alone():
    import bench

    # A rank other than 0 exits at once: no oracle, no data, no output line.
    assert bench.reference_arm(None, rank=1, world=2) == 0


def test_bench_reads_its_rank_from_the_environment(monkeypatch):
    # torchrun's variables name the rank; the reference arm of rank 1 prints nothing.
    import sys

    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.main() == 0
