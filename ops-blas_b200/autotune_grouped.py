"""Autotuner for the grouped factor + solve launch (aclblasSgetrfGetrsGroupedBatched).

For each size bucket it times every candidate configuration of the persistent kernel on a
synthetic batch whose orders are spread uniformly over the bucket (A ~ N(0,1), one right-hand
side), keeps the fastest, and writes the table that aclblasSgetrfGetrsGroupedPlanCreate reads:

    # n_lo n_hi lanes warps rows
    1 4 4 0 0
    ...

Candidates: n <= 16 -- lanes per matrix {natural segment, 32}; 33 <= n <= 128 -- the instantiated
register shapes (rows per lane, warps per matrix) with 32 * rows >= n: (2,2), (2,4), (2,8), (3,4),
(3,8), (4,8); a 2- or 4-warp shape puts four or two matrices in one CTA. Every candidate computes the same bits, so only time
decides. Usage (needs a B200):

    python ops-blas_b200/autotune_grouped.py [--out PATH] [--reps 7]
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SMALL_BUCKETS = [(1, 4), (5, 8), (9, 12), (13, 16), (17, 24), (25, 32)]
MEDIUM_BUCKETS = [(33, 48), (49, 64), (65, 80), (81, 96), (97, 112), (113, 128)]


def _package():
    name = "ops_blas_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _natural(n):
    return 4 if n <= 4 else (8 if n <= 8 else (16 if n <= 16 else 32))


def candidates(lo, hi):
    if hi <= 32:
        return [(_natural(hi), 0, 0)] + ([(32, 0, 0)] if hi <= 16 else [])
    rmin = (hi + 31) // 32
    shapes = [(2, 2), (2, 4), (2, 8), (3, 4), (3, 8), (4, 8)]  # (rows per lane, warps) instantiated
    return [(0, w, r) for r, w in shapes if r >= rmin]


def time_bucket(ob, handle, lo, hi, config, reps, seed=0, target_bytes=256 << 20, max_instances=400_000):
    """Median time (ms) and matrices/s of one grouped execution over a bucket batch."""
    import torch

    ns = list(range(lo, hi + 1))
    mean_bytes = np.mean([4 * n * n for n in ns])
    per = max(8, min(int(target_bytes / mean_bytes / len(ns)), max_instances // len(ns)))
    sizes = [per] * len(ns)
    nrhss = [1] * len(ns)
    plan = ob.GroupedPlan(handle, ns, nrhss, sizes, config=[config] * len(ns))
    used = plan.config()
    a_offs, a_tot = ob.grouped_offsets(ns, ns, ns, sizes)
    b_offs, b_tot = ob.grouped_offsets(ns, nrhss, ns, sizes)
    g = torch.Generator(device="cuda").manual_seed(seed)
    A0 = torch.randn(a_tot, device="cuda", generator=g)
    B0 = torch.randn(b_tot, device="cuda", generator=g)
    A, B = A0.clone(), B0.clone()
    ap, bp = ob.slab_ptrs(A, a_offs), ob.slab_ptrs(B, b_offs)
    piv = torch.empty(sum(n * s for n, s in zip(ns, sizes)), dtype=torch.int32, device="cuda")
    info = torch.empty(sum(sizes), dtype=torch.int32, device="cuda")
    times = []
    for r in range(reps + 2):
        A.copy_(A0)
        B.copy_(B0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.run(handle, ap, piv, info, bp)
        e1.record()
        torch.cuda.synchronize()
        if r >= 2:
            times.append(e0.elapsed_time(e1))
    plan.close()
    ms = float(np.median(times))
    return ms, sum(sizes) / (ms * 1e-3), used[0]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=os.path.join(HERE, "grouped_tuning.txt"))
    ap.add_argument("--reps", type=int, default=7)
    args = ap.parse_args(argv)
    import torch

    ob = _package()
    # time the built-in choices, not a table left from an earlier run
    os.environ["OPSBLAS_GROUPED_TUNING"] = os.devnull
    handle = ob.Handle()
    lines = ["# grouped getrf+getrs tuning table, written by autotune_grouped.py on "
             + torch.cuda.get_device_name(0),
             "# n_lo n_hi lanes warps rows   (candidate: matrices/s)"]
    for lo, hi in SMALL_BUCKETS + MEDIUM_BUCKETS:
        results = {}
        for cfg in candidates(lo, hi):
            ms, rate, used = time_bucket(ob, handle, lo, hi, cfg, args.reps)
            results[tuple(used)] = max(results.get(tuple(used), 0.0), rate)
        best = max(results, key=results.get)
        note = "  ".join(f"{c}:{r:.3e}" for c, r in sorted(results.items()))
        lines.append(f"{lo} {hi} {best[0]} {best[1]} {best[2]}   # {note}")
        print(lines[-1], flush=True)
    handle.close()
    with open(args.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote", args.out)


if __name__ == "__main__":
    main()
