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
import json
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
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


def test_reference_arm_matches_the_gpu_arm_config():
    """The reference arm factors the GPU arm's own inputs (same generator and seed) and reports the
    same config object, so the two lines describe one workload."""
    bench = _bench()
    a1, b1 = bench.chain_inputs(1000, batch=64)
    a2, b2 = bench.chain_inputs(1000, batch=64)
    assert a1.dtype == np.float32 and b1.dtype == np.float32
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    assert a1.shape == (64, bench.N, bench.N) and b1.shape == (64, bench.NRHS, bench.N)
    assert float(b1.min()) >= -1.0 and float(b1.max()) < 1.0
    assert bench.workload_config(1) == bench.workload_config(1)
    assert bench.workload_config(1)["batch_per_gpu"] == bench.BATCH


def test_metric_summary_carries_every_ratio():
    bench = _bench()
    kern = {"getrf": {"frac_hbm": 0.41}}
    plain = {"matrices_s": 1.0e5, "berr_max": 1.2e-7}
    mixed = {"plain": plain, "tf32": {"vs_plain": 2.1, "berr_max": 1.1e-7, "iters_max": 0},
             "bf16": {"vs_plain": 1.6, "berr_max": 9e-7, "iters_max": 1}}
    sections = {"grouped": {"speedup_vs_plain": 1.7, "ms": {"plain": 12.0, "grouped_graph": 7.0, "grouped": 7.1},
                            "grouped_matrices_s": 7e6, "plain_matrices_s": 4e6, "roofline": {"frac": 0.07}},
                "mixed_refine": {"n256_b2048": mixed, "n512_b256": mixed},
                "adjoint": {"fwd_bwd_matrices_s": 9.6e6}}
    s = bench.metric_summary(kern, sections)
    assert s["getrf_frac_hbm"] == 0.41
    assert s["grouped"]["speedup_vs_plain"] == 1.7
    assert s["grouped"]["graph_speedup_vs_plain"] == pytest.approx(12.0 / 7.0, rel=1e-3)
    for n in ("n256", "n512"):
        assert s[f"mixed_{n}"]["tf32"]["vs_plain"] == 2.1
        assert s[f"mixed_{n}"]["plain_berr"] == 1.2e-7
        assert s[f"mixed_{n}"]["bf16"]["berr"] == 9e-7
    assert len(json.dumps(s)) < 1500  # stays inside the tail of the bench's output
