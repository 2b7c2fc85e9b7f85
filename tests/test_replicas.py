"""The N > 1 path of bench.py: one process per GPU running independent
replicas, the device time taken as the max over ranks and the job's rate as
all ranks' steps over it; the reference arm runs on rank 0 alone. Covered
here with two gloo ranks on the CPU (there is no data-path collective to
test: the replicas share nothing)."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, times, results) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.slowest_over_ranks(times[rank], dist, "cpu")
        results[rank] = (slowest, bench.whole_job_rate(world, 30, slowest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_replicas():
    world, port = 2, _free_port()
    times = [41.5, 57.25]
    manager = mp.Manager()
    results = manager.dict()
    mp.spawn(_rank, args=(world, port, times, results), nprocs=world, join=True)
    for rank in range(world):
        slowest, rate = results[rank]
        assert slowest == 57.25
        assert rate == pytest.approx(2 * 30 * 1000.0 / 57.25)


def test_one_process_needs_no_group():
    assert bench.slowest_over_ranks(12.0, None, "cpu") == 12.0
    assert bench.whole_job_rate(1, 30, 60.0) == pytest.approx(500.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    # A rank other than 0 leaves at once, printing nothing; rank 0 is the one
    # that times the CPU reference.
    monkeypatch.setenv("RANK", "1")

    class Args:
        steps, warmup, gpus, reference_warmup = 1, 0, 2, False

    assert bench.reference_arm(Args()) is None
    assert capsys.readouterr().out == ""
