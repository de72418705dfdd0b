#!/usr/bin/env python
"""Benchmark of the batched LU chain on B200.

Workload (one step): the plain FP32 chain at scale -- n = lda = 32, 131072 matrices,
aclblasSgetrfBatched -> aclblasSgetrsBatched (trans N, nrhs = 4) -> aclblasSgetriBatched,
A i.i.d. N(0,1), B i.i.d. U(-1,1), synthetic and seeded. Every step factors its own fresh
copy of the inputs (getrf works in place), so each step reads 512 MiB of matrices that are
not in L2 (126 MB) when the step starts; no L2 flush is needed.

  value       matrices/s of the whole chain, device time, inputs resident in HBM;
  e2e         the same through the C ABI from pinned host buffers: H2D of A and B, the chain,
              D2H of X, inv(A) and info inside the timed region, the batch in 16 chunks over
              three streams so that both copy directions and the chain overlap;
  roofline    the dominant kernel's algorithmic bytes per launch / its CUDA-event duration,
              against the measured HBM copy bandwidth (MEASURED_PEAKS.json);
  cpu_baseline  the reference's CPU golden path (LAPACK through its test headers, built in
              oracle/_ref) on a bounded sample, all host threads.

--impl reference times that CPU golden path alone on the same workload (rank 0 only).
Multi-GPU (torchrun): replicas only -- every rank runs its own batch, no collective on the
data path; value = all ranks' matrices / max-over-ranks time.

sections (single GPU, skipped with --no-sections): grouped uneven batch vs per-n launches,
mixed precision + refinement vs plain FP32, adjoint, fused matinv, geqrf, gels and complex GEMM;
--section NAME
[--small] runs one of them alone.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "getrf+getrs batched matrices/s: mixed/grouped vs plain FP32 at equal FP64 err"
N, BATCH, NRHS = 32, 131072, 4
E2E_CHUNKS = 16  # e2e leg: chunks of the batch, pipelined over E2E_STREAMS streams
E2E_STREAMS = 3
FALLBACK_HBM_GBS = 6650.0
DATA = "synthetic seeded: A ~ N(0,1), B ~ U(-1,1); fresh input copy per step, inputs (512 MiB) > L2"

# Algorithmic bytes per matrix (reads + writes of each kernel):
#   getrf  8n^2 + 4n + 12          A read and written, pivots, info, pointer
#   getrs  4n^2 + 4n + 8n*nrhs + 16  LU read, pivots, B read and written, two pointers
#   getri  8n^2 + 4n + 20          LU read, C written, pivots, info, two pointers
ALG_BYTES = {
    "getrf": 8 * N * N + 4 * N + 12,
    "getrs": 4 * N * N + 4 * N + 8 * N * NRHS + 16,
    "getri": 8 * N * N + 4 * N + 20,
}
FLOPS = {"getrf": 2 * N ** 3 / 3, "getrs": 2 * N * N * NRHS, "getri": 4 * N ** 3 / 3}


def load_package():
    name = "ops_blas_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "ops-blas_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of each kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while the timed region runs."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
    }

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self.nv:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons - {"gpu_idle"}), "samples": len(self.samples)}


def chain_inputs(seed, batch=BATCH):
    """The workload's inputs on the host: A (batch, N, N) i.i.d. N(0,1) and B (batch, NRHS, N) i.i.d.
    U(-1,1), float32, column-major per matrix, from numpy's PCG64 seeded with `seed`. The GPU arm
    and the reference arm factor these same bytes."""
    import numpy as np

    rng = np.random.default_rng(seed)
    a = rng.standard_normal((batch, N, N), dtype=np.float32)
    b = rng.random((batch, NRHS, N), dtype=np.float32) * np.float32(2) - np.float32(1)
    return a, b


def workload_config(world):
    """The config object of both arms' JSON lines."""
    return {"workload": "lu_chain_n32_b131072", "n": N, "lda": N, "batch_per_gpu": BATCH, "nrhs": NRHS,
            "ops": "getrf+getrs(N)+getri", "parallelism": f"replicas{world}", "seed": "1000 + rank",
            "l2": "inputs larger than L2"}


def cpu_reference_rate(a0, b0, nthreads=0, reps=1):
    """Matrices/s of the reference's CPU golden chain (getrf, getrs N nrhs=4, getri) over the host
    matrices a0 / b0 (fresh copies each rep, best of reps); all host threads by default."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import oracle as O

    n_sample = a0.shape[0]
    best = None
    for _ in range(reps):
        lu, x = a0.copy(), b0.copy()
        c = np.empty_like(a0)
        t0 = time.perf_counter()
        piv, _ = O.ref_getrf(lu, N, N, True, nthreads)
        O.ref_getrs("N", lu, N, N, piv, x, NRHS, N, nthreads)
        O.ref_getri(lu, N, N, piv, c, N, nthreads)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    cores = O.ref().ref_max_threads() if nthreads <= 0 else nthreads
    return n_sample / best, cores, O.ref().ref_openblas_config().decode()


def cpu_baseline(a0, b0, reps=3):
    """The reference golden chain on the workload's own host inputs (the whole batch), best of reps."""
    rate, cores, cfg = cpu_reference_rate(a0, b0, reps=reps)
    return {"value": rate, "unit": "matrices/s", "cores": cores, "kind": "reference",
            "sample": f"the workload's own {a0.shape[0]} n=32 matrices (same bytes as the GPU arm), best of {reps}, "
                      f"getrf+getrs(nrhs=4)+getri, reference golden headers over {cfg}, OpenMP over batch chunks"}


def run_reference_arm(args, rank):
    """The reference's CPU golden path timed on the workload itself: every step factors fresh copies
    of the same 131072 matrices the GPU arm factors (same generator and seed), all host threads."""
    if rank != 0:
        return None
    sys.path.insert(0, ROOT)
    import oracle as O

    if O.ref() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/librefgold.so (the reference's CPU "
                                                               "golden path) was not built on this machine"}))
        return None
    a0, b0 = chain_inputs(1000 + rank)
    for _ in range(args.warmup):
        cpu_reference_rate(a0, b0)
    times = []
    cores, cfg = 0, ""
    for _ in range(args.steps):
        r, cores, cfg = cpu_reference_rate(a0, b0)
        times.append(BATCH / r)
    total = sum(times)
    value = BATCH * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": DATA,
        "config": workload_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": "matrices/s", "cores": cores, "kind": "reference",
                         "sample": f"all {BATCH} matrices per step, reference golden headers over {cfg}"},
        "e2e": {"value": value, "unit": "matrices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return line


def max_over_ranks(x, dist=None, device=None):
    """The maximum of x over all ranks (every rank gets it); x itself without a process group."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(matrices_per_rank, world, steps, ms):
    """Matrices/s of the whole job: every rank's matrices over the slowest rank's time."""
    return matrices_per_rank * world * steps / (ms * 1e-3)


def _events_ms(fn, reps, prep=None):
    """Median device time (ms) of fn() over reps runs, prep() outside the timed region."""
    import torch

    ts = []
    for r in range(reps + 1):
        if prep:
            prep()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        if r:
            ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def _fp64_berr(A, X, B):
    """max over matrices and columns of ||b - A x||inf / (||A||inf ||x||inf + ||b||inf), FP64 on the GPU;
    A (batch, n, n), X/B (batch, nrhs, n) in the column-major batch convention."""
    a = A.double().transpose(1, 2)
    x = X.double().transpose(1, 2)
    b = B.double().transpose(1, 2)
    r = b - a @ x
    an = a.abs().sum(2).amax(1)
    return float((r.abs().amax(1) / (an[:, None] * x.abs().amax(1) + b.abs().amax(1))).amax())


def cpu_solve_rate(ns, nrhs, seed=7):
    """Matrices/s of the reference's CPU golden getrf + getrs (trans N) over the orders in ns (one
    matrix per entry, grouped by order), all host threads; returns (rate, cores, seconds)."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import oracle as O

    rng = np.random.default_rng(seed)
    groups = {}
    for n in ns:
        groups[n] = groups.get(n, 0) + 1
    data = [(n, rng.standard_normal((c, n, n)).astype(np.float32), rng.standard_normal((c, nrhs, n)).astype(np.float32))
            for n, c in groups.items()]
    t0 = time.perf_counter()
    for n, a, b in data:
        piv, _ = O.ref_getrf(a, n, n, True, 0)
        O.ref_getrs("N", a, n, n, piv, b, nrhs, n, 0)
    dt = time.perf_counter() - t0
    return len(ns) / dt, O.ref().ref_max_threads(), dt


def cpu_section_baseline(ns, nrhs, what, target_s=3.0):
    """cpu_solve_rate on a sample sized to about target_s seconds, as a cpu_baseline object."""
    probe = list(ns[: max(1, min(len(ns), 16))])
    rate, cores, dt = cpu_solve_rate(probe, nrhs)
    k = int(max(1, min(len(ns), rate * target_s)))
    rate, cores, dt = cpu_solve_rate(list(ns[:k]), nrhs)
    return {"value": rate, "unit": "matrices/s", "cores": cores, "kind": "reference",
            "sample": f"{k} matrices of {what}: reference golden getrf + getrs(N) (LAPACK through its test headers), "
                      f"OpenMP over batch chunks, {dt:.1f} s"}


def section_grouped(ob, h, dev, peak, reps=5, instances=50000):
    """Configuration 3: 50000 instances, n ~ U{4..128}, nrhs = 1, one persistent launch (direct and
    replayed from a CUDA graph) against the plain path (per-n getrf + getrs launches)."""
    import numpy as np
    import torch

    rng = np.random.default_rng(0)
    nv = rng.integers(4, 129, size=instances)
    ns = sorted(set(int(v) for v in nv), reverse=True)
    sizes = [int((nv == n).sum()) for n in ns]
    nrhss = [1] * len(ns)
    a_offs, a_tot = ob.grouped_offsets(ns, ns, ns, sizes)
    b_offs, b_tot = ob.grouped_offsets(ns, nrhss, ns, sizes)
    g = torch.Generator(device=dev).manual_seed(3)
    A0 = torch.randn(a_tot, device=dev, generator=g)
    B0 = torch.randn(b_tot, device=dev, generator=g)
    A, B = A0.clone(), B0.clone()
    ap, bp = ob.slab_ptrs(A, a_offs), ob.slab_ptrs(B, b_offs)
    piv = torch.empty(sum(n * s for n, s in zip(ns, sizes)), dtype=torch.int32, device=dev)
    info = torch.empty(sum(sizes), dtype=torch.int32, device=dev)
    s = torch.cuda.Stream(device=dev)
    hs = ob.Handle(stream=s)
    plan = ob.GroupedPlan(hs, ns, nrhss, sizes)
    prep = lambda: (A.copy_(A0), B.copy_(B0))
    with torch.cuda.stream(s):
        t_grp = _events_ms(lambda: plan.run(hs, ap, piv, info, bp), reps, prep)
        assert int(info.max()) == 0
        t_plain = _events_ms(lambda: ob.grouped_plain(hs, ns, nrhss, sizes, ns, ns, ap, piv, info, bp), reps, prep)
        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=s):
            plan.run(hs, ap, piv, info, bp)
        t_graph = _events_ms(graph.replay, reps, prep)
    del graph
    plan.close()
    hs.close()
    total = sum(sizes)
    alg = sum(sz * (12 * n * n + 16 * n + 28) for n, sz in zip(ns, sizes))
    return {"workload": f"grouped_{instances}_n4-128_nrhs1", "instances": total,
            "grouped_matrices_s": total / (t_grp * 1e-3), "grouped_graph_matrices_s": total / (t_graph * 1e-3),
            "plain_matrices_s": total / (t_plain * 1e-3), "speedup_vs_plain": t_plain / min(t_grp, t_graph),
            "ms": {"grouped": t_grp, "grouped_graph": t_graph, "plain": t_plain},
            "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved_GB_s": alg / (min(t_grp, t_graph) * 1e-3) / 1e9,
                         "frac": alg / (min(t_grp, t_graph) * 1e-3) / 1e9 / peak},
            "GFLOP_s": sum(sz * (2 * n ** 3 / 3 + 2 * n * n) for n, sz in zip(ns, sizes)) / (min(t_grp, t_graph) * 1e-3) / 1e9,
            "plain_path": "per-n aclblasSgetrfBatched + aclblasSgetrsBatched",
            "cpu_baseline": cpu_section_baseline([int(v) for v in nv], 1, "the same n ~ U{4..128} draw, nrhs = 1")}

def section_mixed(ob, h, dev, reps=3, sizes=((256, 2048), (512, 256))):
    """Configuration 4: kappa = 1e4 (A = Q1 diag(logspace(0,4)) Q2^T in FP64, stored FP32), B ~ N(0,1),
    nrhs = 16. Plain FP32 getrf + getrs against factor + solve + FP64-residual refinement with the
    TF32 and BF16 split trailing updates; every result's backward error is measured in FP64."""
    import torch

    out = {}
    for n, batch in sizes:
        g = torch.Generator(device=dev).manual_seed(n)
        q1, _ = torch.linalg.qr(torch.randn(batch, n, n, device=dev, dtype=torch.float64, generator=g))
        q2, _ = torch.linalg.qr(torch.randn(batch, n, n, device=dev, dtype=torch.float64, generator=g))
        sv = torch.logspace(0, 4, n, device=dev, dtype=torch.float64)
        A32 = ((q1 * sv) @ q2.transpose(1, 2)).transpose(1, 2).contiguous().float()
        del q1, q2
        B = torch.randn(batch, 16, n, device=dev, generator=g)
        LU, X = torch.empty_like(A32), torch.empty_like(B)
        pa, px = ob.ptr_array(LU), ob.ptr_array(X)
        piv = torch.empty((batch, n), dtype=torch.int32, device=dev)
        info = torch.empty(batch, dtype=torch.int32, device=dev)

        def plain():
            LU.copy_(A32)
            X.copy_(B)
            h.getrf(LU, n, n, piv=piv, info=info, aptr=pa)
            h.getrs("N", LU, n, n, piv, X, 16, n, aptr=pa, bptr=px)

        t_plain = _events_ms(plain, reps)
        res = {"plain": {"matrices_s": batch / (t_plain * 1e-3), "ms": t_plain, "berr_max": _fp64_berr(A32, X, B)}}
        for name, comp in (("tf32", ob.COMPUTE_32F_FAST_TF32), ("bf16", ob.COMPUTE_32F_FAST_16BF)):
            box = {}
            t = _events_ms(lambda: box.update(r=h.refine(A32, B, n, 16, compute=comp, max_iter=10, tol=1e-6)), reps)
            Xm, _, _, _, _, it = box["r"]
            res[name] = {"matrices_s": batch / (t * 1e-3), "ms": t, "berr_max": _fp64_berr(A32, Xm, B),
                         "iters_max": int(it.max()), "vs_plain": t_plain / t}
        fl = 2 * n ** 3 / 3 + 2 * n * n * 16
        for v in res.values():
            v["GFLOP_s"] = fl * v["matrices_s"] / 1e9
            v["alg_GB_s"] = (12 * n * n + 8 * n * 16) * v["matrices_s"] / 1e9
        res["cpu_baseline"] = cpu_section_baseline([n] * batch, 16, f"n = {n}, nrhs = 16, N(0,1)")
        out[f"n{n}_b{batch}"] = res
        del A32, B, LU, X
        torch.cuda.empty_cache()
    return out


def section_adjoint(ob, h, dev, reps=3, batch=65536):
    """Configuration 5: X = A^{-1} B with A = G + 8 I, n = 64, nrhs = 8, 65536 matrices; forward
    getrf + getrs and the adjoint (dB = A^{-T} dX by the transposed solve on the stored factors,
    dA = -dB X^T by the batched GEMM)."""
    import torch

    n, nrhs = 64, 8
    g = torch.Generator(device=dev).manual_seed(5)
    A = torch.randn(batch, n, n, device=dev, generator=g) + 8 * torch.eye(n, device=dev)
    B = torch.randn(batch, nrhs, n, device=dev, generator=g)
    dX0 = torch.randn(batch, nrhs, n, device=dev, generator=g)
    LU, X, dX, dA = torch.empty_like(A), torch.empty_like(B), torch.empty_like(dX0), torch.empty_like(A)
    pa, px = ob.ptr_array(LU), ob.ptr_array(X)
    piv = torch.empty((batch, n), dtype=torch.int32, device=dev)
    info = torch.empty(batch, dtype=torch.int32, device=dev)

    def fwd():
        LU.copy_(A)
        X.copy_(B)
        h.getrf(LU, n, n, piv=piv, info=info, aptr=pa)
        h.getrs("N", LU, n, n, piv, X, nrhs, n, aptr=pa, bptr=px)

    def bwd():
        dX.copy_(dX0)
        h.adjoint(LU, n, n, piv, X, n, dX, n, dA, n)

    t_f = _events_ms(fwd, reps)
    t_b = _events_ms(bwd, reps)
    return {"workload": f"adjoint_n64_nrhs8_b{batch}", "forward_matrices_s": batch / (t_f * 1e-3),
            "backward_matrices_s": batch / (t_b * 1e-3), "fwd_bwd_matrices_s": batch / ((t_f + t_b) * 1e-3),
            "ms": {"forward": t_f, "backward": t_b},
            "GFLOP_s_forward": (2 * n ** 3 / 3 + 2 * n * n * nrhs) * batch / (t_f * 1e-3) / 1e9,
            "cpu_baseline_forward": cpu_section_baseline([n] * batch, nrhs, "n = 64, nrhs = 8, N(0,1) (the reference has no adjoint)")}

def section_matinv(ob, h, dev, peak, reps=5, batch=131072):
    """aclblasSmatinvBatched at the chain's shape, n = 32 (512 MiB of input, larger than L2): the
    fused launch against the two-call sequence the reference's matinv runs -- a copy of A,
    aclblasSgetrfBatched on it, aclblasSgetriBatched into Ainv."""
    import torch

    n = 32
    g = torch.Generator(device=dev).manual_seed(7)
    A = torch.randn(batch, n, n, device=dev, generator=g)
    Ainv, LU = torch.empty_like(A), torch.empty_like(A)
    pa, pc, pl = ob.ptr_array(A), ob.ptr_array(Ainv), ob.ptr_array(LU)
    piv = torch.empty((batch, n), dtype=torch.int32, device=dev)
    info = torch.empty(batch, dtype=torch.int32, device=dev)
    finfo = torch.empty(batch, dtype=torch.int32, device=dev)

    def fused():
        h.matinv(A, n, n, Ainv, n, info=info, aptr=pa, cptr=pc)

    def two_call():
        LU.copy_(A)
        h.getrf(LU, n, n, piv=piv, info=finfo, aptr=pl)
        h.getri(LU, n, n, piv, Ainv, n, info=info, aptr=pl, cptr=pc)

    t_f = _events_ms(fused, reps)
    t_s = _events_ms(two_call, reps)
    alg = (8 * n * n + 20) * batch  # A read, Ainv written, info, two pointers
    return {"workload": f"matinv_n32_b{batch}", "fused_matrices_s": batch / (t_f * 1e-3),
            "two_call_matrices_s": batch / (t_s * 1e-3), "speedup_vs_two_call": t_s / t_f,
            "ms": {"fused": t_f, "two_call": t_s},
            "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved_GB_s": alg / (t_f * 1e-3) / 1e9,
                         "frac": alg / (t_f * 1e-3) / 1e9 / peak},
            "two_call_note": "copy of A + getrf + getri, the reference matinv's device sequence"}


def section_geqrf(ob, h, dev, peak, reps=5, batch=131072):
    """aclblasSgeqrfBatched at the chain's shape, 32 x 32 (512 MiB of input, larger than L2):
    in-place Householder QR, tau out."""
    import torch

    m = n = 32
    g = torch.Generator(device=dev).manual_seed(9)
    A0 = torch.randn(batch, n, m, device=dev, generator=g)
    A = torch.empty_like(A0)
    tau = torch.empty(batch, n, device=dev)
    pa, pt = ob.ptr_array(A), ob.ptr_array(tau)
    t = _events_ms(lambda: h.geqrf(A, m, n, m, tau=tau, aptr=pa, tptr=pt), reps, prep=lambda: A.copy_(A0))
    alg = (8 * m * n + 4 * n + 16) * batch  # A read and written, tau, two pointers
    return {"workload": f"geqrf_32x32_b{batch}", "matrices_s": batch / (t * 1e-3), "ms": t,
            "GFLOP_s": (2 * m * n * n - 2 * n ** 3 / 3) * batch / (t * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved_GB_s": alg / (t * 1e-3) / 1e9,
                         "frac": alg / (t * 1e-3) / 1e9 / peak}}


def section_gels(ob, h, dev, peak, reps=5, batch=65536):
    """aclblasSgelsBatched, least squares 32 x 16 with 2 right-hand sides (overdetermined, the
    QR path), inputs in HBM: A read and written, C read and written."""
    import torch

    m, n, nrhs = 32, 16, 2
    g = torch.Generator(device=dev).manual_seed(13)
    A0 = torch.randn(batch, n, m, device=dev, generator=g)
    C0 = torch.randn(batch, nrhs, m, device=dev, generator=g)
    A, Cm = torch.empty_like(A0), torch.empty_like(C0)
    pa, pc = ob.ptr_array(A), ob.ptr_array(Cm)
    info = torch.empty(batch, dtype=torch.int32, device=dev)

    def prep():
        A.copy_(A0)
        Cm.copy_(C0)

    t = _events_ms(lambda: h.gels("N", A, m, n, nrhs, m, Cm, m, info=info, aptr=pa, cptr=pc), reps, prep=prep)
    alg = (8 * m * n + 8 * m * nrhs + 4 + 16) * batch
    return {"workload": f"gels_32x16_nrhs2_b{batch}", "matrices_s": batch / (t * 1e-3), "ms": t,
            "roofline": {"bound": "hbm", "alg_bytes": alg, "achieved_GB_s": alg / (t * 1e-3) / 1e9,
                         "frac": alg / (t * 1e-3) / 1e9 / peak},
            "note": "warp per system (M >= N, M <= 32, N + nrhs <= 32), serial row-order sums"}


# FP32 FMA peak of the CUDA cores: 148 SMs x 128 lanes x 2 FLOP x 1965 MHz (nominal; not measured)
FP32_SIMT_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def section_cgemm(ob, h, dev, reps=5, batch=16384):
    """aclblasCgemmBatched, 64 x 64 x 64 complex, alpha and beta complex (C read and written),
    inputs in HBM (1.5 GiB, larger than L2). FP32 CUDA-core bound: 8 m n k FLOP per matrix.
    Beside it, for context: torch.bmm on complex64 tensors of the same shape (cuBLAS), and the
    reference golden's BLAS (scipy's OpenBLAS cgemm, one thread) on a host sample."""
    import time

    import torch

    m = n = k = 64
    g = torch.Generator(device=dev).manual_seed(17)
    A = torch.randn((batch, k, m), dtype=torch.complex64, device=dev, generator=g)
    B = torch.randn((batch, n, k), dtype=torch.complex64, device=dev, generator=g)
    Cm = torch.randn((batch, n, m), dtype=torch.complex64, device=dev, generator=g)
    pa, pb, pc = ob.ptr_array(A), ob.ptr_array(B), ob.ptr_array(Cm)
    alpha, beta = 1.5 + 0.3j, 0.3 - 0.1j
    t = _events_ms(lambda: h.cgemm("N", "N", m, n, k, alpha, A, m, B, k, beta, Cm, m, aptr=pa, bptr=pb, cptr=pc),
                   reps)
    D = torch.empty_like(Cm)
    t_lib = _events_ms(lambda: torch.bmm(B, A, out=D), reps)  # (A B)^T = B^T A^T in row-major storage
    flop = 8.0 * m * n * k * batch
    out = {"workload": f"cgemm_64x64x64_b{batch}", "matrices_s": batch / (t * 1e-3), "ms": t,
           "GFLOP_s": flop / (t * 1e-3) / 1e9,
           "roofline": {"bound": "fp32_simt", "achieved_TFLOP_s": flop / (t * 1e-3) / 1e12,
                        "peak_TFLOP_s": FP32_SIMT_TFLOPS, "frac": flop / (t * 1e-3) / 1e12 / FP32_SIMT_TFLOPS,
                        "peak_note": "nominal 148 SMs x 128 FP32 lanes x 2 x 1965 MHz"},
           "torch_bmm_complex64_ms": t_lib,
           "torch_bmm_note": "cuBLAS complex GEMM of the same shape without alpha/beta, for context"}
    try:
        import numpy as np
        from threadpoolctl import threadpool_limits

        sys.path.insert(0, ROOT)
        import oracle as O

        ns = 2048
        rng = np.random.default_rng(0)
        a = (rng.standard_normal((ns, k, m)) + 1j * rng.standard_normal((ns, k, m))).astype(np.complex64)
        b = (rng.standard_normal((ns, n, k)) + 1j * rng.standard_normal((ns, n, k))).astype(np.complex64)
        c = (rng.standard_normal((ns, n, m)) + 1j * rng.standard_normal((ns, n, m))).astype(np.complex64)
        with threadpool_limits(limits=1):
            t0 = time.perf_counter()
            O.ref_cgemm("N", "N", m, n, k, alpha, a, m, b, k, beta, c, m)
            dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": ns / dt, "unit": "matrices/s", "cores": 1, "kind": "reference",
                               "sample": f"{ns} matrices 64x64x64: the reference golden's cblas_cgemm (scipy "
                                         f"OpenBLAS, one thread), {dt:.2f} s"}
    except Exception as e:  # the baseline is reported, never required
        out["cpu_baseline"] = {"value": None, "unavailable": str(e)[:200]}
    return out


def section_chain(ob, h, dev, peak, reps=5, batch=BATCH):
    """The headline chain (getrf -> getrs nrhs 4 -> getri at n = 32) on `batch` matrices, each kernel
    timed on its own over fresh input copies; --small runs 32768 matrices (128 MiB, still larger
    than L2) for profiling captures."""
    import torch

    a, b = chain_inputs(1000, batch)
    A0, B0 = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    A, B, Cinv = torch.empty_like(A0), torch.empty_like(B0), torch.empty_like(A0)
    pa, pb, pc = ob.ptr_array(A), ob.ptr_array(B), ob.ptr_array(Cinv)
    piv = torch.empty((batch, N), dtype=torch.int32, device=dev)
    info = torch.empty(batch, dtype=torch.int32, device=dev)
    rinfo = torch.empty(batch, dtype=torch.int32, device=dev)
    prep = lambda: (A.copy_(A0), B.copy_(B0))
    t_f = _events_ms(lambda: h.getrf(A, N, N, piv=piv, info=info, aptr=pa), reps, prep)
    t_s = _events_ms(lambda: h.getrs("N", A, N, N, piv, B, NRHS, N, aptr=pa, bptr=pb), reps, lambda: B.copy_(B0))
    t_i = _events_ms(lambda: h.getri(A, N, N, piv, Cinv, N, info=rinfo, aptr=pa, cptr=pc), reps)
    out = {"workload": f"lu_chain_n32_b{batch}"}
    for k, t in (("getrf", t_f), ("getrs", t_s), ("getri", t_i)):
        gbs = ALG_BYTES[k] * batch / (t * 1e-3) / 1e9
        out[k] = {"ms": t, "GB_s": gbs, "frac_hbm": gbs / peak}
    return out


def section_gemm(ob, h, dev, reps=5, batch=2048, size=256):
    """aclblasGemmBatchedEx on the tcgen05 tensor cores: size^3 per matrix, BF16 -> BF16, FP16 ->
    FP16 and FP8 E4M3 -> FP16 (FP32 accumulation), plus FP32 with FAST_TF32; alpha = 1, beta = 0.
    TFLOP/s against the measured cuBLAS BF16 peak (MEASURED_PEAKS.json); torch.bmm of the same
    shape for context (BF16 / FP16)."""
    import torch

    m = n = k = size
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16_peak, peak_kind = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        bf16_peak, peak_kind = 1590.0, "fallback"
    g = torch.Generator(device=dev).manual_seed(19)
    out = {"workload": f"gemm_batched_{size}^3_b{batch}", "peak_bf16_TFLOP_s": bf16_peak, "peak_source": peak_kind}
    flop = 2.0 * m * n * k * batch
    cases = (("bf16", torch.bfloat16, ob.ACL_BF16, torch.bfloat16, ob.ACL_BF16, ob.COMPUTE_32F),
             ("f16", torch.float16, ob.ACL_FLOAT16, torch.float16, ob.ACL_FLOAT16, ob.COMPUTE_32F),
             ("e4m3", torch.float8_e4m3fn, ob.ACL_FLOAT8_E4M3FN, torch.float16, ob.ACL_FLOAT16, ob.COMPUTE_32F),
             ("tf32", torch.float32, ob.ACL_FLOAT, torch.float32, ob.ACL_FLOAT, ob.COMPUTE_32F_FAST_TF32))
    for name, tin, ain, tout, aout, comp in cases:
        ta_ = "T" if name == "tf32" else "N"  # FP32 operands arrive by TMA when K-contiguous
        A = torch.randn((batch, k, m), device=dev, generator=g).to(tin)  # m == k: either orientation
        B = torch.randn((batch, n, k), device=dev, generator=g).to(tin)
        Cm = torch.zeros((batch, n, m), device=dev, dtype=tout)
        pa, pb, pc = ob.ptr_array(A), ob.ptr_array(B), ob.ptr_array(Cm)
        t = _events_ms(lambda: h.gemm_batched_ex(ta_, "N", m, n, k, 1.0, A, ain, m, B, ain, k, 0.0, Cm, aout, m,
                                                 compute=comp, aptr=pa, bptr=pb, cptr=pc), reps)
        e_ = {"op": ta_ + "N"}
        e = {**e_, "ms": t, "TFLOP_s": flop / (t * 1e-3) / 1e12,
             "frac_of_bf16_peak": flop / (t * 1e-3) / 1e12 / bf16_peak}
        if name in ("bf16", "f16"):
            D = torch.empty_like(Cm)
            e["torch_bmm_ms"] = _events_ms(lambda: torch.bmm(B, A, out=D), reps)
        out[name] = e
        del A, B, Cm
    return out


def run_section(args):
    """One measured section on its own (used for profiling captures with --small)."""
    import torch

    dev = torch.device("cuda", 0)
    ob = load_package()
    h = ob.Handle()
    peak, _ = peaks()
    if args.section == "gemm":
        out = section_gemm(ob, h, dev, reps=2 if args.small else 5, batch=256 if args.small else 2048)
    elif args.section == "chain":
        out = section_chain(ob, h, dev, peak, reps=2 if args.small else 5, batch=32768 if args.small else BATCH)
    elif args.section == "grouped":
        out = section_grouped(ob, h, dev, peak, reps=2, instances=5000 if args.small else 50000)
    elif args.section == "mixed":
        out = section_mixed(ob, h, dev, reps=2, sizes=((256, 148), (512, 160)) if args.small else ((256, 2048), (512, 256)))
    elif args.section == "gels":
        out = section_gels(ob, h, dev, peak, reps=2, batch=16384 if args.small else 65536)
    elif args.section == "geqrf":
        out = section_geqrf(ob, h, dev, peak, reps=2, batch=65536 if args.small else 131072)
    elif args.section == "matinv":
        out = section_matinv(ob, h, dev, peak, reps=2, batch=65536 if args.small else 131072)
    elif args.section == "cgemm":
        out = section_cgemm(ob, h, dev, reps=2, batch=4096 if args.small else 16384)
    else:
        out = section_adjoint(ob, h, dev, reps=2, batch=8192 if args.small else 65536)
    print(json.dumps({"section": args.section, "small": bool(args.small), **out}))
    h.close()


def _r(x, d=4):
    """x rounded to d significant digits (compact JSON)."""
    return None if x is None else float(f"{x:.{d}g}")


def metric_summary(kern, sections):
    """The metric's own ratios (grouped and mixed + refinement against the plain FP32 path, with the
    FP64 backward errors of both arms) and the headline kernel's HBM fraction, compact, as the last
    key of the JSON line."""
    out = {"getrf_frac_hbm": _r(kern["getrf"]["frac_hbm"], 3)}
    g = sections.get("grouped")
    if g:
        out["grouped"] = {"speedup_vs_plain": _r(g["speedup_vs_plain"]),
                          "graph_speedup_vs_plain": _r(g["ms"]["plain"] / g["ms"]["grouped_graph"]),
                          "matrices_s": _r(g["grouped_matrices_s"]), "plain_matrices_s": _r(g["plain_matrices_s"]),
                          "frac_hbm": _r(g["roofline"]["frac"], 3)}
    m = sections.get("mixed_refine") or {}
    for key, v in m.items():
        n = key.split("_")[0]
        e = {"plain_berr": _r(v["plain"]["berr_max"], 3), "plain_matrices_s": _r(v["plain"]["matrices_s"])}
        for p in ("tf32", "bf16"):
            if p in v:
                e[p] = {"vs_plain": _r(v[p]["vs_plain"]), "berr": _r(v[p]["berr_max"], 3), "iters": v[p]["iters_max"]}
        out[f"mixed_{n}"] = e
    a = sections.get("adjoint")
    if a:
        out["adjoint_fwd_bwd_matrices_s"] = _r(a["fwd_bwd_matrices_s"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sections", action="store_true", help="skip the section measurements (grouped, mixed, adjoint, matinv, geqrf, gels, cgemm)")
    ap.add_argument("--section", choices=["chain", "gemm", "grouped", "mixed", "adjoint", "matinv", "geqrf", "gels", "cgemm"],
                    help="run only this measured section (one JSON line) and exit")
    ap.add_argument("--small", action="store_true", help="with --section: reduced sizes (profiling captures)")
    args = ap.parse_args()
    assert args.warmup >= 3 or args.impl == "reference" or os.environ.get("OPSBLAS_BENCH_ALLOW_SHORT"), \
        "at least 3 warm-up steps"

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.section:
        run_section(args)
        return

    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ob = load_package()
    h = ob.Handle()
    stream = torch.cuda.current_stream()

    nbuf = args.warmup + args.steps
    a_host, b_host = chain_inputs(1000 + rank)
    A_first = torch.from_numpy(a_host).to(dev)
    B_first = torch.from_numpy(b_host).to(dev)
    # one fresh device copy of the inputs per step (getrf and getrs work in place)
    A0 = [A_first.clone() for _ in range(nbuf)]
    B0 = [B_first.clone() for _ in range(nbuf)]
    del A_first, B_first
    aptr = [ob.ptr_array(a) for a in A0]
    bptr = [ob.ptr_array(b) for b in B0]
    Cinv = torch.empty((BATCH, N, N), device=dev)
    cptr = ob.ptr_array(Cinv)
    piv = torch.empty((BATCH, N), dtype=torch.int32, device=dev)
    info = torch.empty(BATCH, dtype=torch.int32, device=dev)
    rinfo = torch.empty(BATCH, dtype=torch.int32, device=dev)

    def step(i, ev=None):
        if ev:
            ev[0].record(stream)
        h.getrf(A0[i], N, N, piv=piv, info=info, aptr=aptr[i])
        if ev:
            ev[1].record(stream)
        h.getrs("N", A0[i], N, N, piv, B0[i], NRHS, N, aptr=aptr[i], bptr=bptr[i])
        if ev:
            ev[2].record(stream)
        h.getri(A0[i], N, N, piv, Cinv, N, info=rinfo, aptr=aptr[i], cptr=cptr)
        if ev:
            ev[3].record(stream)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    assert int(info.max()) == 0 and int(rinfo.max()) == 0

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        start.record(stream)
        for s in range(args.steps):
            step(args.warmup + s, evs[s])
        stop.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(stop)
    per = {"getrf": [], "getrs": [], "getri": []}
    for e in evs:
        per["getrf"].append(e[0].elapsed_time(e[1]))
        per["getrs"].append(e[1].elapsed_time(e[2]))
        per["getri"].append(e[2].elapsed_time(e[3]))
    ms = max_over_ranks(ms, dist, dev)

    # e2e through the C ABI from pinned host memory
    hostA = torch.empty((BATCH, N, N), dtype=torch.float32).pin_memory()
    hostB = torch.empty((BATCH, NRHS, N), dtype=torch.float32).pin_memory()
    hostA.copy_(torch.from_numpy(a_host))
    hostB.copy_(torch.from_numpy(b_host))
    hostX = torch.empty_like(hostB).pin_memory()
    hostC = torch.empty_like(hostA).pin_memory()
    hostI = torch.empty(BATCH, dtype=torch.int32).pin_memory()
    dA, dB = A0[0], B0[0]
    # The batch goes through in E2E_CHUNKS chunks round-robin over three streams (one handle
    # each), so the host-to-device copy of one chunk, the chain of the previous one and the
    # device-to-host copy of the one before run at the same time (PCIe is full duplex).
    e2e_streams = [torch.cuda.Stream(dev) for _ in range(E2E_STREAMS)]
    e2e_handles = [ob.Handle(stream=s_) for s_ in e2e_streams]
    per_chunk = (BATCH + E2E_CHUNKS - 1) // E2E_CHUNKS

    def e2e_step():
        head = torch.cuda.Event()
        head.record(stream)
        for s_ in e2e_streams:
            s_.wait_event(head)
        for c in range(E2E_CHUNKS):
            i0, i1 = c * per_chunk, min(BATCH, (c + 1) * per_chunk)
            if i0 >= i1:
                break
            s_, hh = e2e_streams[c % E2E_STREAMS], e2e_handles[c % E2E_STREAMS]
            with torch.cuda.stream(s_):
                a_, b_, ap, bp = dA[i0:i1], dB[i0:i1], aptr[0][i0:i1], bptr[0][i0:i1]
                a_.copy_(hostA[i0:i1], non_blocking=True)
                b_.copy_(hostB[i0:i1], non_blocking=True)
                hh.getrf(a_, N, N, piv=piv[i0:i1], info=info[i0:i1], aptr=ap)
                hh.getrs("N", a_, N, N, piv[i0:i1], b_, NRHS, N, aptr=ap, bptr=bp)
                hh.getri(a_, N, N, piv[i0:i1], Cinv[i0:i1], N, info=rinfo[i0:i1], aptr=ap, cptr=cptr[i0:i1])
                hostX[i0:i1].copy_(b_, non_blocking=True)
                hostC[i0:i1].copy_(Cinv[i0:i1], non_blocking=True)
                hostI[i0:i1].copy_(rinfo[i0:i1], non_blocking=True)
        for s_ in e2e_streams:
            tail = torch.cuda.Event()
            tail.record(s_)
            stream.wait_event(tail)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    assert int(hostI.max()) == 0
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, dist, dev)
    h2d = hostA.numel() * 4 + hostB.numel() * 4
    d2h = hostX.numel() * 4 + hostC.numel() * 4 + hostI.numel() * 4

    if rank == 0:
        peak, peak_kind = peaks()
        tot = {k: sum(v) for k, v in per.items()}
        dom = max(tot, key=tot.get)
        kern = {}
        for k, v in per.items():
            avg = sum(v) / len(v)
            gbs = ALG_BYTES[k] * BATCH / (avg * 1e-3) / 1e9
            kern[k] = {"ms_avg": avg, "GB_s": gbs, "frac_hbm": gbs / peak,
                       "GFLOP_s": FLOPS[k] * BATCH / (avg * 1e-3) / 1e9}
        traffic = profiled_traffic().get(dom)
        line = {
            "metric": METRIC,
            "value": whole_job_rate(BATCH, world, args.steps, ms),
            "unit": "matrices/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": DATA,
            "config": workload_config(world),
            "kernels": kern,
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": kern[dom]["GB_s"], "peak": peak,
                         "unit": "GB/s", "frac": kern[dom]["frac_hbm"], "peak_source": peak_kind,
                         "traffic": traffic, "alg_bytes_per_launch": ALG_BYTES[dom] * BATCH},
            "e2e": {"value": BATCH * world / (e2e_ms * 1e-3), "unit": "matrices/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                    "pipeline": f"{E2E_CHUNKS} chunks over {E2E_STREAMS} streams"},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(a_host, b_host)
            except Exception as e:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "unavailable": str(e)[:200]}
        if world == 1 and not args.no_sections:
            sections = {"grouped": section_grouped(ob, h, dev, peak), "mixed_refine": section_mixed(ob, h, dev),
                        "adjoint": section_adjoint(ob, h, dev), "matinv": section_matinv(ob, h, dev, peak),
                        "geqrf": section_geqrf(ob, h, dev, peak), "gels": section_gels(ob, h, dev, peak),
                        "cgemm": section_cgemm(ob, h, dev), "gemm": section_gemm(ob, h, dev)}
            # the full sections on a line of their own (not JSON: the JSON line below stays the only one)
            print("sections " + json.dumps(sections))
            line["metric_summary"] = metric_summary(kern, sections)
        print(json.dumps(line))
    h.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
