"""The bench's multi-rank host logic on CPU: two gloo ranks (one replica each)
agree on the slowest rank's time and on the whole-job aggregate, and the
reference arm runs on rank 0 only."""

from __future__ import annotations

import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(0.5 + 0.25 * rank, torch.device("cpu"))
        out[rank] = (t, bench.whole_job_mlups(world, 1000, 10, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    t, value = res[0]
    assert t == 0.75
    assert abs(value - 2 * 1000 * 10 / 0.75 / 1e6) < 1e-12


def test_single_process_is_a_no_op():
    import bench

    assert bench.max_over_ranks(1.25, torch.device("cpu")) == 1.25
    assert bench.whole_job_mlups(1, 10, 5, 2.0) == 25e-6


def test_reference_arm_only_on_rank_zero(monkeypatch, capsys):
    import argparse

    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    bench.run_reference(argparse.Namespace(steps=1, warmup=0))
    assert capsys.readouterr().out == ""
