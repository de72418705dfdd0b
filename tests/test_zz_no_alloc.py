"""GPU test of aclblasSgetrfsRefineBatchedStaticScratch, the refinement entry point whose scratch is
a fixed device array instead of the handle workspace. Calls in a row (different sizes, compute
types and data, so each finds the previous call's leftovers in the scratch) are compared with
aclblasSgetrfsRefineBatchedEx on the same inputs. Both run the same kernels in the same order, so
every output -- factors, pivots, info, iteration counts, X and the backward errors -- must be
equal bit for bit. One case has n = 400, where the residual kernel needs more than 48 KiB of
shared memory (the set-up the entry point does on its first call per device). The file name keeps
it last in collection, after every other GPU test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import to_dev, to_host

pytestmark = pytest.mark.gpu


def _inputs(n, nrhs, batch, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    b = rng.standard_normal((batch, nrhs, n)).astype(np.float32)
    return a, b


def _static_call(ob, handle, A, B, n, nrhs, compute, max_iter, tol):
    import torch

    batch = A.shape[0]
    LU = torch.empty_like(A)
    X = torch.empty_like(B)
    piv = torch.empty((batch, n), dtype=torch.int32, device=A.device)
    info = torch.empty(batch, dtype=torch.int32, device=A.device)
    berr = torch.empty(batch, dtype=torch.float64, device=A.device)
    iters = torch.empty(batch, dtype=torch.int32, device=A.device)
    pa, plu, pb, px = ob.ptr_array(A), ob.ptr_array(LU), ob.ptr_array(B), ob.ptr_array(X)
    st = ob.lib().aclblasSgetrfsRefineBatchedStaticScratch(
        handle.h, n, nrhs, pa.data_ptr(), n, plu.data_ptr(), n, piv.data_ptr(), pb.data_ptr(), n, px.data_ptr(), n,
        compute, max_iter, tol, berr.data_ptr(), iters.data_ptr(), info.data_ptr(), batch)
    return st, (X, LU, piv, info, berr, iters, pa, plu, pb, px)


def _small_buffers(torch, count):
    """count small real device buffers (never written: the calls below are rejected first)."""
    return [torch.zeros(64, dtype=torch.float64, device="cuda") for _ in range(count)]


@pytest.mark.parametrize("n,nrhs,batch", [
    (64, 64, (8 << 20) // (((64 * 64 * 4 + 255) // 256) * 256 + 20) + 1),  # the batch's scratch is too large
    (4096, 600, 1),  # one matrix's correction block alone is larger than the scratch
])
def test_oversize_request_is_rejected(ob, handle, n, nrhs, batch):
    """A request whose scratch exceeds the static array fails before any launch."""
    import torch

    bufs = _small_buffers(torch, 9)
    P = [C.c_void_p(t.data_ptr()) for t in bufs]
    st = ob.lib().aclblasSgetrfsRefineBatchedStaticScratch(
        handle.h, n, nrhs, P[0], n, P[1], n, P[2], P[3], n, P[4], n, ob.COMPUTE_32F_FAST_TF32, 5, 1e-6, P[5], P[6],
        P[7], batch)
    torch.cuda.synchronize()
    assert st == ob.INVALID_VALUE
    assert all(float(t.abs().sum()) == 0.0 for t in bufs)


def test_static_scratch_matches_workspace_entry_point(ob, handle):
    import torch

    cases = [  # (n, nrhs, batch, computeType, maxIter, seed)
        (48, 4, 512, ob.COMPUTE_32F_FAST_TF32, 10, 11),
        (20, 2, 1000, ob.COMPUTE_32F, 3, 12),
        (400, 4, 6, ob.COMPUTE_32F_FAST_TF32, 2, 13),
    ]
    data = [(_inputs(n, nrhs, batch, seed), n, nrhs, comp, it) for n, nrhs, batch, comp, it, seed in cases]
    tol = 1e-6
    results = []
    for (a, b), n, nrhs, comp, it in data:  # two calls in a row, nothing in between
        A, B = to_dev(a, "cuda"), to_dev(b, "cuda")
        st, out = _static_call(ob, handle, A, B, n, nrhs, comp, it, tol)
        assert st == ob.SUCCESS
        results.append((A, B, out))
    torch.cuda.synchronize()
    for ((a, b), n, nrhs, comp, it), (A, B, out) in zip(data, results):
        X, LU, piv, info, berr, iters = out[:6]
        rX, rLU, rpiv, rinfo, rberr, riters = handle.refine(A, B, n, nrhs, compute=comp, max_iter=it, tol=tol)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(to_host(piv), to_host(rpiv))
        np.testing.assert_array_equal(to_host(info), to_host(rinfo))
        np.testing.assert_array_equal(to_host(iters), to_host(riters))
        assert np.array_equal(to_host(LU).view(np.uint32), to_host(rLU).view(np.uint32))
        assert np.array_equal(to_host(X).view(np.uint32), to_host(rX).view(np.uint32))
        assert np.array_equal(to_host(berr).view(np.uint64), to_host(rberr).view(np.uint64))
        # inputs untouched
        assert np.array_equal(to_host(A), a) and np.array_equal(to_host(B), b)
