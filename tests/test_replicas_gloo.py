"""Multi-process path of bench.py on CPU: world_size-2 `gloo` process group.

The engine runs replicas only (one independent solve per GPU, no data-path
collective); the one collective of the N > 1 bench is the all-reduce MAX of
the ranks' device times, which gives the whole-job rate.  These tests run it
with two CPU processes, and check that the reference arm's non-zero ranks do
no work.
"""
from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank                      # rank 1 is the slow one
        ms_max, rate = bench.replica_rate(ms, 1000, world)
        dist.barrier()
        results[rank] = (ms_max, rate)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_rate_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        results = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(90)
            assert p.exitcode == 0
        got = dict(results)
    assert set(got) == {0, 1}
    for ms_max, rate in got.values():
        assert ms_max == 150.0                        # the slowest rank's time, on every rank
        assert rate == pytest.approx(2 * 1000 / 0.150)


def test_single_rank_rate_needs_no_process_group():
    import bench

    assert bench.replica_rate(250.0, 500, 1) == (250.0, pytest.approx(2000.0))


def test_reference_arm_nonzero_rank_does_no_work(capsys):
    import bench

    bench.run_reference_arm(None, 1, 2)               # returns before touching its arguments
    assert capsys.readouterr().out == ""
