"""GPU test of aclblasSgetrfsRefineBatchedStaticScratch, the refinement entry point whose scratch is
a fixed device array instead of the handle workspace. Two calls in a row (different sizes, compute
types and data, so the second finds the first's leftovers in the scratch) are compared with
aclblasSgetrfsRefineBatchedEx on the same inputs. Both run the same kernels, so the factors,
pivots, info and iteration counts must be equal; X and the backward errors within 1e-6
relative. The file name keeps it last in collection, after every other GPU test.
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


def test_oversize_request_is_rejected(ob, handle):
    """A batch whose scratch exceeds the static array fails before any launch."""
    n, nrhs = 64, 64
    per = ((n * nrhs * 4 + 255) // 256) * 256 + 20
    batch = (8 << 20) // per + 1
    P = C.c_void_p(0x1000)  # never dereferenced: the size check comes first
    st = ob.lib().aclblasSgetrfsRefineBatchedStaticScratch(
        handle.h, n, nrhs, P, n, P, n, P, P, n, P, n, ob.COMPUTE_32F_FAST_TF32, 5, 1e-6, P, P, P, batch)
    assert st == ob.INVALID_VALUE


def test_static_scratch_matches_workspace_entry_point(ob, handle):
    import torch

    cases = [  # (n, nrhs, batch, computeType, maxIter, seed)
        (48, 4, 512, ob.COMPUTE_32F_FAST_TF32, 10, 11),
        (20, 2, 1000, ob.COMPUTE_32F, 3, 12),
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
        np.testing.assert_allclose(to_host(X), to_host(rX), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(to_host(berr), to_host(rberr), rtol=1e-6, atol=1e-12)
        # inputs untouched
        assert np.array_equal(to_host(A), a) and np.array_equal(to_host(B), b)
