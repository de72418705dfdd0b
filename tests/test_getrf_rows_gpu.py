"""GPU parity of aclblasSgetrfBatched's blocked path for 128 < n <= 1024 (getrf_blocked_tc.cu):
the matrix transposed in place to rows, 32-column panels with the whole-row interchanges applied
once per panel, the tiled trailing update, the transpose back. Every element takes the reference's
updates one fmaf at a time in the reference's order, so factors, pivots and info must equal the
CPU oracle (the reference's unblocked kernel restated) bit for bit, including stops at zero
pivots inside later panels, the no-pivot mode, row strides that are not a multiple of four (the
element-wise paths) and the fallback kernel taken when the handle has no workspace."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from conftest import to_dev, to_host
from test_lu_gpu import assert_bitwise, gpu_getrf

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,lda", [(257, 257), (320, 323), (512, 512), (545, 548), (1024, 1024)])
def test_blocked_rows_bitwise(handle, n, lda):
    """Pivoted factorisation of N(0,1) matrices (padding beyond n untouched)."""
    rng = np.random.default_rng(n + lda)
    batch = 3
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    a[:, :, n:] = 4321.0
    lu, piv, info = gpu_getrf(handle, a, n, lda)
    olu = a.copy()
    opiv, oinfo, _ = O.port_getrf(olu, n, lda)
    assert_bitwise(lu, olu, f"LU n={n}")
    np.testing.assert_array_equal(piv, opiv)
    np.testing.assert_array_equal(info, oinfo)
    assert np.all(lu[:, :, n:] == 4321.0)


def test_blocked_rows_stops_in_later_panels(handle):
    """Zero columns at 0, 31, 32, 100 and 299 (first column of a panel, last column of a panel,
    inside a later panel, the last column): info, the zeroed trailing pivots and the partially
    factored matrices match the reference's stop semantics bit for bit."""
    n, batch = 300, 6
    rng = np.random.default_rng(17)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    for q, col in enumerate([0, 31, 32, 100, 299]):
        a[q, col, :] = 0.0  # column col (column-major batch convention)
    lu, piv, info = gpu_getrf(handle, a, n, n)
    olu = a.copy()
    opiv, oinfo, _ = O.port_getrf(olu, n, n)
    assert_bitwise(lu, olu, "LU")
    np.testing.assert_array_equal(piv, opiv)
    np.testing.assert_array_equal(info, oinfo)
    assert list(info[:5]) == [1, 32, 33, 101, 300] and info[5] == 0


@pytest.mark.parametrize("n", [200, 384])
def test_blocked_rows_no_pivot(handle, ob, n):
    """PivotArray == NULL and infoArray == NULL: the reference's no-pivot variant."""
    import torch

    rng = np.random.default_rng(n)
    batch = 4
    a = (rng.standard_normal((batch, n, n)) + 3 * n * np.eye(n)).astype(np.float32)
    A = to_dev(a, "cuda")
    aptr = ob.ptr_array(A)
    assert ob.lib().aclblasSgetrfBatched(handle.h, n, aptr.data_ptr(), n, None, None, batch) == ob.SUCCESS
    torch.cuda.synchronize()
    olu = a.copy()
    O.port_getrf(olu, n, n, pivot=False)
    assert_bitwise(to_host(A), olu, "LU")


def test_blocked_rows_without_workspace_falls_back_bit_identical(ob):
    """With a 16-byte workspace the blocked path's four bytes per matrix (20 here) are missing:
    the call takes the one-CTA-per-matrix kernel, whose results are the same bits."""
    import torch

    n, batch = 300, 5
    rng = np.random.default_rng(23)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    ws = torch.zeros(16, dtype=torch.uint8, device="cuda")
    h = ob.Handle()
    try:
        assert ob.lib().aclblasSetWorkspace(h.h, C.c_void_p(ws.data_ptr()), C.c_size_t(16)) == ob.SUCCESS
        lu0, piv0, info0 = gpu_getrf(h, a, n, n)
    finally:
        h.close()
    h2 = ob.Handle()
    try:
        lu1, piv1, info1 = gpu_getrf(h2, a, n, n)
    finally:
        h2.close()
    torch.cuda.synchronize()
    assert_bitwise(lu0, lu1, "LU")
    np.testing.assert_array_equal(piv0, piv1)
    np.testing.assert_array_equal(info0, info1)
