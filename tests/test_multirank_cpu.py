"""The multi-rank path of bench.py on CPU: two gloo ranks (world size 2, 127.0.0.1).

bench.py runs one replica per GPU (every matrix is independent, no collective on the data path);
the only cross-rank steps are the barriers around the timed region and the max-over-ranks time.
These tests run exactly those helpers on two CPU processes, and check that rank 1 of the
reference arm exits without printing (rank 0 alone reports).
"""
from __future__ import annotations

import importlib.util
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")  # per-rank times 10 and 15 ms
        rate = bench.whole_job_rate(1000, world, 4, ms)
        dist.barrier()
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 15.0  # the slowest rank's time on every rank
        assert rate == pytest.approx(1000 * 2 * 4 / 15e-3)


def test_helpers_without_a_process_group():
    bench = _bench()
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.whole_job_rate(131072, 1, 20, 20.0) == pytest.approx(131072 * 1000.0)


def test_reference_arm_other_ranks_print_nothing():
    bench = _bench()

    class Args:
        steps, warmup = 1, 0

    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference_arm(Args, 1) is None
    assert buf.getvalue() == ""
