"""Multi-rank logic of bench.py on CPU (gloo, two ranks).

The engine does not shard one lattice: under torchrun every rank advances
its own replica, and the only collectives are a barrier and the max of the
per-rank device times.  These tests run that reduction over a real two-rank
gloo process group and check the whole-job figure and the reference arm's
rank handling.
"""

import io
import os
import socket
from contextlib import redirect_stdout

import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank          # rank 1 is the slower replica
        ms = bench.max_over_ranks(local_ms, dist, "cpu")
        dist.barrier()
        out.put((rank, ms, bench.whole_job_mlups(1000, world, 20, ms / 1e3)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, q), nprocs=2, join=True, start_method="spawn")
    got = sorted(q.get() for _ in range(2))
    for rank, ms, value in got:
        assert ms == 15.0                      # every rank reports the slowest replica
        assert value == pytest.approx(1000 * 2 * 20 / 0.015 / 1e6)


def test_without_process_group_value_is_local():
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.whole_job_mlups(10, 1, 5, 2.0) == pytest.approx(25e-6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    buf = io.StringIO()
    with redirect_stdout(buf):
        rc = bench.run_reference(None, dict(bench.WORKLOADS["sphere512"]))
    assert rc == 0 and buf.getvalue() == ""
