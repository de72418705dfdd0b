"""Pins the CPU oracle (this project's C restatement of the reference kernels) against the
reference's own golden path: the committed fixtures of tests/golden/ (made from the reference's
LAPACK-backed golden headers by tests/golden/gen_golden.py) and, where oracle/_ref was built,
the golden path itself run live on the reference's CSV cases.

Criteria are the reference tests' own (sgetrf_batched_test.cpp:206-258, getrs_batched_test.cpp:
232-262, sgetri_batched_test.cpp:118-150): info exact; pivots exact (here: for matrices whose
pivot choices are untied, relative top-2 gap >= 1e-5); factors, solutions and inverses under
the FP32 MIXED_TOLERANCE rule, skipped for singular matrices; plus a 1e-5 normwise bound.
"""
from __future__ import annotations

import os
import zlib

import numpy as np
import pytest

import oracle as O
from cases import GETRF, GETRI, GETRS

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TIE = 1e-5
NORMWISE = 1e-5


def crc(a):
    return zlib.crc32(np.ascontiguousarray(a).tobytes())


def c1_inputs():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((1024, 16, 16)).astype(np.float32)
    B = rng.standard_normal((1024, 1, 16)).astype(np.float32)
    return A, B


def block(a, rows, cols):
    return a[:, :cols, :rows]


def solution_ok(x, x_gold, A, b):
    """Solution parity between two FP32 LU solvers. The north-star 1e-5 normwise bound is what
    two backward-stable solvers can promise only up to the conditioning of A: they may differ
    by up to ~kappa_2(A) * 2^-24 in the forward error. So: normwise difference <= max(1e-5,
    2 * kappa_2(A) * 2^-24), and backward error at most twice the golden solution's."""
    M = A.T.astype(np.float64)
    kappa = np.linalg.cond(M)
    rel = O.normwise_rel(x, x_gold)
    if rel > max(NORMWISE, 2.0 * kappa * 2.0 ** -24):
        return False
    return O.backward_error(M, x, b) <= 2.0 * O.backward_error(M, x_gold, b) + 2.0 ** -24


def test_c1_fixture_inputs_reproduce():
    g = np.load(os.path.join(GOLD, "c1.npz"))
    A, B = c1_inputs()
    assert crc(A) == int(g["crcA"]) and crc(B) == int(g["crcB"])


def test_c1_oracle_matches_golden():
    g = np.load(os.path.join(GOLD, "c1.npz"))
    A, B = c1_inputs()
    lu = A.copy()
    piv, info, gap = O.port_getrf(lu, 16, 16)
    np.testing.assert_array_equal(info, g["info"])
    untied = gap >= TIE
    assert untied.sum() >= 1000  # N(0,1) data: near-ties are rare
    np.testing.assert_array_equal(piv[untied], g["piv"][untied])
    k = len(g["LU"])
    for b in range(k):
        assert O.mixed_tolerance_ok(lu[b], g["LU"][b])
        assert O.normwise_rel(lu[b], g["LU"][b]) <= NORMWISE
    x = B.copy()
    O.port_getrs("N", lu, 16, 16, piv, x, 1, 16)
    for b in range(1024):
        if g["info"][b] == 0:
            assert solution_ok(x[b].T, g["X"][b].T, A[b], B[b].T), b


def _fixture():
    return np.load(os.path.join(GOLD, "csv_small.npz"))


@pytest.mark.parametrize("c", [c for c in GETRF if c.status == "SUCCESS" and c.n > 0 and c.batch > 0
                               and c.n <= 32], ids=lambda c: c.name)
def test_getrf_fixture(c):
    g = _fixture()
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    assert crc(a) == int(g[f"getrf/{c.name}/crc"])
    piv, info, gap = O.port_getrf(a, c.n, c.lda, c.pivot)
    np.testing.assert_array_equal(info, g[f"getrf/{c.name}/info"])
    if c.pivot:
        gp = g[f"getrf/{c.name}/piv"]
        for b in range(c.batch):
            if gap[b] >= TIE or info[b] > 0:
                np.testing.assert_array_equal(piv[b], gp[b])
    glu = g[f"getrf/{c.name}/lu"]
    for b in range(len(glu)):
        if info[b] == 0:
            assert O.mixed_tolerance_ok(block(a[b:b + 1], c.n, c.n), block(glu[b:b + 1], c.n, c.n))


@pytest.mark.parametrize("c", [c for c in GETRS if c.status == "SUCCESS" and c.n > 0 and c.batch > 0
                               and c.nrhs > 0 and c.n <= 32], ids=lambda c: c.name)
def test_getrs_fixture(c):
    g = _fixture()
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    b = O.case_rhs(c.n, c.nrhs, c.ldb, c.seed, c.batch)
    assert [crc(a), crc(b)] == list(g[f"getrs/{c.name}/crc"])
    piv, info = O.ref_getrf_for_solve(a, c.n, c.lda, c.pivot) if O.ref() else (None, None)
    if piv is None and c.pivot:
        pytest.skip("the reference golden library is needed to factor the solve inputs")
    O.port_getrs(c.trans, a, c.n, c.lda, piv if c.pivot else None, b, c.nrhs, c.ldb)
    gx = g[f"getrs/{c.name}/x"]
    rf = g[f"getrs/{c.name}/rfinfo"]
    for k in range(c.batch):
        if rf[k] == 0:
            assert O.mixed_tolerance_ok(block(b[k:k + 1], c.n, c.nrhs), block(gx[k:k + 1], c.n, c.nrhs)), k


@pytest.mark.parametrize("c", [c for c in GETRI if c.status == "SUCCESS" and c.n > 0 and c.batch > 0
                               and c.n <= 32], ids=lambda c: c.name)
def test_getri_fixture(c):
    if O.ref() is None:
        pytest.skip("the reference golden library is needed to factor the inverse inputs")
    g = _fixture()
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    assert crc(a) == int(g[f"getri/{c.name}/crc"])
    piv, _ = O.ref_getrf_for_solve(a, c.n, c.lda, c.pivot)
    cc = np.zeros((c.batch, c.n, c.ldc), np.float32)
    info = O.port_getri(a, c.n, c.lda, piv if c.pivot else None, cc, c.ldc)
    ginfo = g[f"getri/{c.name}/info"]
    # The reference kernel reports the highest zero diagonal, LAPACK the lowest; they agree
    # whenever at most one diagonal entry is zero, which holds for every CSV case.
    np.testing.assert_array_equal(info, ginfo)
    gc = g[f"getri/{c.name}/c"]
    for k in range(len(gc)):
        if ginfo[k] == 0:
            assert O.mixed_tolerance_ok(block(cc[k:k + 1], c.n, c.n), block(gc[k:k + 1], c.n, c.n)), k


# ------------------------------------------------------------ live pin against oracle/_ref --

needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref (reference golden path) not built here")
SMALL_WORK = 600_000_000  # n^3 * batch bound that keeps the CPU suite within a few minutes


@needs_ref
@pytest.mark.parametrize("c", [c for c in GETRF if c.status == "SUCCESS" and c.n > 0 and c.batch > 0],
                         ids=lambda c: c.name)
def test_getrf_live_vs_reference(c):
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    ref = a.copy()
    piv, info, gap = O.port_getrf(a, c.n, c.lda, c.pivot)
    rpiv, rinfo = O.ref_getrf(ref, c.n, c.lda, c.pivot)
    np.testing.assert_array_equal(info, rinfo)
    for b in range(c.batch):
        if c.pivot and (gap[b] >= TIE or info[b] > 0):
            np.testing.assert_array_equal(piv[b], rpiv[b])
        if info[b] == 0:
            x, y = block(a[b:b + 1], c.n, c.n), block(ref[b:b + 1], c.n, c.n)
            assert O.mixed_tolerance_ok(x, y)
            assert O.normwise_rel(x, y) <= NORMWISE


@needs_ref
@pytest.mark.parametrize("c", [c for c in GETRS if c.status == "SUCCESS" and c.n > 0 and c.batch > 0
                               and c.nrhs > 0 and c.n ** 2 * c.batch * c.nrhs < SMALL_WORK], ids=lambda c: c.name)
def test_getrs_live_vs_reference(c):
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    b = O.case_rhs(c.n, c.nrhs, c.ldb, c.seed, c.batch)
    piv, rf = O.ref_getrf_for_solve(a, c.n, c.lda, c.pivot)
    x, y = b.copy(), b.copy()
    O.port_getrs(c.trans, a, c.n, c.lda, piv if c.pivot else None, x, c.nrhs, c.ldb)
    O.ref_getrs(c.trans, a, c.n, c.lda, piv if c.pivot else None, y, c.nrhs, c.ldb)
    for k in range(c.batch):
        if rf[k] == 0:
            assert O.mixed_tolerance_ok(block(x[k:k + 1], c.n, c.nrhs), block(y[k:k + 1], c.n, c.nrhs)), k


@needs_ref
@pytest.mark.parametrize("c", [c for c in GETRI if c.status == "SUCCESS" and c.n > 0 and c.batch > 0
                               and c.n ** 3 * c.batch < SMALL_WORK], ids=lambda c: c.name)
def test_getri_live_vs_reference(c):
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    piv, _ = O.ref_getrf_for_solve(a, c.n, c.lda, c.pivot)
    x = np.zeros((c.batch, c.n, c.ldc), np.float32)
    y = np.zeros_like(x)
    info = O.port_getri(a, c.n, c.lda, piv if c.pivot else None, x, c.ldc)
    rinfo = O.ref_getri(a, c.n, c.lda, piv if c.pivot else None, y, c.ldc)
    np.testing.assert_array_equal(info, rinfo)
    for k in range(c.batch):
        if rinfo[k] == 0:
            # The reference test zeroes |v| < 1e-6 on both sides before comparing
            # (sgetri_batched_test.cpp:131-139).
            xs = np.where(np.abs(x[k]) < 1e-6, 0, x[k])[None]
            ys = np.where(np.abs(y[k]) < 1e-6, 0, y[k])[None]
            assert O.mixed_tolerance_ok(block(xs, c.n, c.n), block(ys, c.n, c.n)), k


def test_oracle_nan_and_zero_pivot_rules():
    """Zero and NaN candidates are never chosen as pivots; an all-zero column picks the
    diagonal and stops with info = col + 1 and the remaining pivots zeroed."""
    a = np.zeros((1, 4, 4), np.float32)
    M = np.array([[0, 1, 2, 3], [np.nan, 5, 6, 7], [0, 9, 1, 1], [2, 1, 1, 5]], np.float32)
    a[0] = M.T
    piv, info, _ = O.port_getrf(a, 4, 4)
    assert piv[0][0] == 4  # |2| beats zeros and NaN
    z = np.zeros((1, 3, 3), np.float32)
    z[0] = np.array([[0, 1, 2], [0, 3, 4], [0, 5, 7]], np.float32).T
    piv, info, _ = O.port_getrf(z, 3, 3)
    assert info[0] == 1 and list(piv[0]) == [1, 0, 0]
