"""bench.py's multi-rank host logic with two gloo ranks on the CPU.

Under torchrun every rank runs an independent replica of the loop (the path does
not shard), so the only cross-rank steps are reductions of times: each rank
reports the slowest rank's time (max over ranks) and the job rate counts every
rank's steps over that time.  The reference arm runs on rank 0 alone; the other
ranks return without work.
"""

import argparse
import datetime
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        mine = [10.0 + rank, 5.0 * (ws - rank), float(rank)]  # times of this rank's replica
        got = bench.max_over_ranks(dist, torch, mine, "cpu")
        q.put((rank, got, bench.job_rate(ws, 100, got[0])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    try:
        res = [q.get(timeout=180) for _ in range(ws)]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(r for r, _, _ in res) == [0, 1]
    for _, got, rate in res:
        assert got == [11.0, 10.0, 1.0]  # every rank sees the slowest rank's times
        assert rate == pytest.approx(2 * 100 / 0.011)  # both ranks' steps over the slowest time


def test_single_process_reduction_is_the_identity():
    import bench

    assert bench.max_over_ranks(None, None, [3.0, 4.5], "cpu") == [3.0, 4.5]
    assert bench.job_rate(1, 50, 100.0) == pytest.approx(500.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = argparse.Namespace(gpus=2, steps=3, warmup=1)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""  # no line, no work
