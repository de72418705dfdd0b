"""GPU tests of the grouped persistent factor + solve (aclblasSgetrfGetrsGrouped*).

Every instance must come out bit-identical to aclblasSgetrfBatched followed by
aclblasSgetrsBatched (trans N) on the same matrix -- LU, pivots, info and X -- whatever the
per-group configuration (lanes per matrix, warps per matrix, rows per lane), over repeated
executions (the persistent kernel resets its own work counters) and when replayed from a CUDA
graph. The plain path itself is pinned to the oracle by test_lu_gpu.py; a sample is checked
against the oracle here too.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import to_host

pytestmark = pytest.mark.gpu


def _setup(ob, ns, nrhss, sizes, seed, ldpad=0, singular=()):
    import torch

    rng = np.random.default_rng(seed)
    ldas = [n + ldpad for n in ns]
    ldbs = [n + ldpad for n in ns]
    a_offs, a_tot = ob.grouped_offsets(ns, ns, ldas, sizes)
    b_offs, b_tot = ob.grouped_offsets(ns, [max(r, 1) for r in nrhss], ldbs, sizes)
    a = rng.standard_normal(a_tot).astype(np.float32)
    b = rng.standard_normal(b_tot).astype(np.float32)
    # make some instances singular: column 0 (or a middle column) of instance i zero
    i = 0
    for g, (n, sz) in enumerate(zip(ns, sizes)):
        for k in range(sz):
            if i in singular and n > 0:
                col = (i % n)
                a[a_offs[i] + col * ldas[g]: a_offs[i] + col * ldas[g] + n] = 0.0
            i += 1
    return dict(ns=ns, nrhss=nrhss, sizes=sizes, ldas=ldas, ldbs=ldbs, a=a, b=b, a_offs=a_offs, b_offs=b_offs,
                total=sum(sizes), piv_total=sum(n * s for n, s in zip(ns, sizes)))


def _device(ob, d):
    import torch

    A = torch.from_numpy(d["a"]).cuda()
    B = torch.from_numpy(d["b"]).cuda()
    piv = torch.full((max(d["piv_total"], 1),), -1, dtype=torch.int32, device="cuda")
    info = torch.full((max(d["total"], 1),), -1, dtype=torch.int32, device="cuda")
    return A, B, ob.slab_ptrs(A, d["a_offs"]), ob.slab_ptrs(B, d["b_offs"]), piv, info


def _run_both(ob, handle, d, config=None, repeats=1):
    import torch

    plan = ob.GroupedPlan(handle, d["ns"], d["nrhss"], d["sizes"], d["ldas"], d["ldbs"], config=config)
    out = []
    for _ in range(repeats):
        A, B, ap, bp, piv, info = _device(ob, d)
        plan.run(handle, ap, piv, info, bp)
        torch.cuda.synchronize()
        out.append((to_host(A), to_host(B), to_host(piv), to_host(info)))
    A, B, ap, bp, piv, info = _device(ob, d)
    ob.grouped_plain(handle, d["ns"], d["nrhss"], d["sizes"], d["ldas"], d["ldbs"], ap, piv, info, bp)
    torch.cuda.synchronize()
    ref = (to_host(A), to_host(B), to_host(piv), to_host(info))
    cfg = plan.config()
    plan.close()
    return out, ref, cfg


def _assert_same(got, ref):
    for x, y in zip(got, ref):
        if x.dtype == np.float32:
            # bitwise, with any NaN matching any NaN (singular instances)
            xn, yn = np.isnan(x), np.isnan(y)
            assert np.array_equal(xn, yn)
            assert np.array_equal(x.view(np.uint32)[~xn], y.view(np.uint32)[~yn])
        else:
            assert np.array_equal(x, y)


MIXED = dict(ns=[1, 2, 3, 4, 5, 7, 8, 9, 13, 16, 17, 24, 31, 32, 33, 40, 47, 48, 64, 65, 90, 100, 127, 128, 130],
             nrhss=[1, 1, 2, 1, 3, 1, 1, 2, 1, 1, 4, 1, 1, 2, 1, 3, 1, 1, 2, 1, 1, 5, 1, 1, 2],
             sizes=[3, 5, 2, 9, 7, 6, 11, 4, 5, 13, 3, 2, 5, 33, 2, 3, 1, 5, 4, 3, 2, 3, 1, 2, 2])


def test_grouped_matches_plain_mixed_sizes(ob, handle):
    d = _setup(ob, **MIXED, seed=1)
    out, ref, _ = _run_both(ob, handle, d)
    _assert_same(out[0], ref)


def test_grouped_repeated_executions_reset_counters(ob, handle):
    d = _setup(ob, **MIXED, seed=2)
    out, ref, _ = _run_both(ob, handle, d, repeats=3)
    for o in out:
        _assert_same(o, ref)


@pytest.mark.parametrize("config", [(32, 0, 0), (0, 2, 2), (0, 4, 2), (0, 8, 2), (0, 4, 3), (0, 8, 3), (0, 8, 4)])
def test_grouped_every_config_gives_the_same_bits(ob, handle, config):
    d = _setup(ob, **MIXED, seed=3, ldpad=3)
    cfgs = [config] * len(d["ns"])
    out, ref, used = _run_both(ob, handle, d, config=cfgs)
    _assert_same(out[0], ref)
    for n, (lanes, warps, rows) in zip(d["ns"], used):
        if n <= 32:
            assert lanes in (4, 8, 16, 32) and (config[0] != 32 or lanes == 32)
        elif n <= 128:  # larger orders run on the batched kernels, their shape is unused
            assert 32 * rows >= n and (rows, warps) in [(2, 2), (2, 4), (2, 8), (3, 4), (3, 8), (4, 8)]
            if config[2] and 32 * config[2] >= n:
                assert (warps, rows) == (config[1], config[2])


def test_grouped_singular_and_factor_only(ob, handle):
    ns = [5, 16, 32, 40, 96, 128]
    d = _setup(ob, ns=ns, nrhss=[1, 0, 2, 1, 0, 1], sizes=[6, 6, 6, 6, 6, 6], seed=4,
               singular=set(range(0, 36, 4)))
    out, ref, _ = _run_both(ob, handle, d)
    _assert_same(out[0], ref)
    info = out[0][3]
    assert (info[0:36:4] > 0).all()


def test_grouped_against_oracle_sample(ob, handle, oracle_mod):
    import torch

    O = oracle_mod
    ns, nrhss, sizes = [6, 20, 50, 77], [1, 2, 1, 3], [4, 3, 3, 2]
    d = _setup(ob, ns=ns, nrhss=nrhss, sizes=sizes, seed=5)
    plan = ob.GroupedPlan(handle, ns, nrhss, sizes)
    A, B, ap, bp, piv, info = _device(ob, d)
    plan.run(handle, ap, piv, info, bp)
    torch.cuda.synchronize()
    a, b, p, inf = to_host(A), to_host(B), to_host(piv), to_host(info)
    i = poff = 0
    for n, nrhs, sz in zip(ns, nrhss, sizes):
        for _ in range(sz):
            m = d["a"][d["a_offs"][i]:d["a_offs"][i] + n * n].reshape(1, n, n).copy()
            opiv, oinfo, _ = O.port_getrf(m, n, n)
            rhs = d["b"][d["b_offs"][i]:d["b_offs"][i] + n * nrhs].reshape(1, nrhs, n).copy()
            O.port_getrs("N", m, n, n, opiv, rhs, nrhs, n)
            got_lu = a[d["a_offs"][i]:d["a_offs"][i] + n * n].reshape(1, n, n)
            got_x = b[d["b_offs"][i]:d["b_offs"][i] + n * nrhs].reshape(1, nrhs, n)
            assert np.array_equal(got_lu.view(np.uint32), m.view(np.uint32))
            assert np.array_equal(got_x.view(np.uint32), rhs.view(np.uint32))
            assert np.array_equal(p[poff:poff + n], opiv.reshape(-1))
            assert inf[i] == int(np.asarray(oinfo).reshape(-1)[0])
            i += 1
            poff += n
    plan.close()


def _gather(flat, offs, span):
    """Instances of one group out of a slab: rows of ``span`` floats at the given offsets."""
    idx = np.asarray(offs, np.int64)[:, None] + np.arange(span, dtype=np.int64)[None, :]
    return flat[idx]


def test_grouped_configuration3_full_draw_against_oracle(ob, handle, oracle_mod):
    """The grouped configuration in full: 50000 instances with n ~ U{4..128} (seed 0), nrhs = 1,
    A and B i.i.d. N(0,1), one persistent launch. Every instance's LU, pivots, info and X equal
    the oracle (the reference's unblocked getrf and trans-N getrs, restated) bit for bit."""
    import torch

    O = oracle_mod
    nv = np.random.default_rng(0).integers(4, 129, size=50000)
    ns = sorted(set(int(v) for v in nv), reverse=True)
    sizes = [int((nv == n).sum()) for n in ns]
    nrhss = [1] * len(ns)
    d = _setup(ob, ns=ns, nrhss=nrhss, sizes=sizes, seed=7)
    plan = ob.GroupedPlan(handle, ns, nrhss, sizes)
    A, B, ap, bp, piv, info = _device(ob, d)
    plan.run(handle, ap, piv, info, bp)
    torch.cuda.synchronize()
    plan.close()
    a, b, p, inf = to_host(A), to_host(B), to_host(piv), to_host(info)
    i = poff = 0
    for n, sz in zip(ns, sizes):
        ao, bo = d["a_offs"][i:i + sz], d["b_offs"][i:i + sz]
        lu = _gather(d["a"], ao, n * n).reshape(sz, n, n)
        x = _gather(d["b"], bo, n).reshape(sz, 1, n)
        opiv, oinfo, _ = O.port_getrf(lu, n, n)
        O.port_getrs("N", lu, n, n, opiv, x, 1, n)
        _assert_same((_gather(a, ao, n * n).reshape(sz, n, n), _gather(b, bo, n).reshape(sz, 1, n),
                      p[poff:poff + sz * n].reshape(sz, n), inf[i:i + sz]),
                     (lu, x, opiv.reshape(sz, n), np.asarray(oinfo).reshape(-1)))
        i += sz
        poff += sz * n
    assert i == 50000


def test_grouped_cuda_graph_replay(ob):
    import torch

    d = _setup(ob, **MIXED, seed=6)
    s = torch.cuda.Stream()
    h = ob.Handle(stream=s)
    plan = ob.GroupedPlan(h, d["ns"], d["nrhss"], d["sizes"], d["ldas"], d["ldbs"])
    A, B, ap, bp, piv, info = _device(ob, d)
    a0, b0 = A.clone(), B.clone()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.run(h, ap, piv, info, bp)
    results = []
    for _ in range(2):
        with torch.cuda.stream(s):
            A.copy_(a0)
            B.copy_(b0)
            g.replay()
        torch.cuda.synchronize()
        results.append((to_host(A), to_host(B), to_host(piv), to_host(info)))
    A2, B2, ap2, bp2, piv2, info2 = _device(ob, d)
    ob.grouped_plain(h, d["ns"], d["nrhss"], d["sizes"], d["ldas"], d["ldbs"], ap2, piv2, info2, bp2)
    torch.cuda.synchronize()
    ref = (to_host(A2), to_host(B2), to_host(piv2), to_host(info2))
    for r in results:
        _assert_same(r, ref)
    del g
    plan.close()
    h.close()


def test_grouped_tuning_table_is_read(ob, handle, tmp_path, monkeypatch):
    table = tmp_path / "t.txt"
    table.write_text("# n_lo n_hi lanes warps rows\n1 16 32 0 0\n33 64 0 4 3\n65 128 0 8 4\n")
    monkeypatch.setenv("OPSBLAS_GROUPED_TUNING", str(table))
    plan = ob.GroupedPlan(handle, [8, 40, 100], [1, 1, 1], [2, 2, 2])
    assert plan.config() == [(32, 0, 0), (0, 4, 3), (0, 8, 4)]
    plan.close()
