"""CPU oracle for the batched LU chain -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
package, and only as the checker. The library (``ops-blas_b200``) never imports it.

Array convention: a batch of column-major ``ld x ncols`` matrices is a C-contiguous float32
numpy array of shape ``(batch, ncols, ld)``; element (i, j) of matrix b is ``arr[b, j, i]``.

* ``port_*``: this project's C restatement of the reference device kernels (lu_oracle.c).
* ``ref_*``: the reference's own CPU golden path (LAPACK through its test headers), available
  where ``oracle/_ref/librefgold.so`` was built.
* ``case_*``: the reference test suites' input generators (case_inputs.cpp).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_oracle as _build

_lib = None
_ref = None

MATRIX_TYPES = {
    "RANDOM_NONSINGULAR": 0,
    "IDENTITY": 1,
    "DIAGONALLY_DOMINANT": 2,
    "ILL_CONDITIONED": 3,
    "DIAGONAL": 4,
    "UPPER_TRIANGULAR": 5,
    "LOWER_TRIANGULAR": 6,
    "SINGULAR_ZERO_COL": 7,
    "SINGULAR_DEPENDENT_ROW": 8,
    "MIXED": 9,
}
TRANS = {"N": 0, "T": 1, "C": 2}
TRANS_ACL = {"N": 111, "T": 112, "C": 113}

_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int)
_f64p = C.POINTER(C.c_double)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def lib():
    global _lib
    if _lib is None:
        path = _build.ORACLE_LIB
        if not os.path.exists(path):
            _build.build_oracle()
        L = C.CDLL(path)
        L.oracle_sgetrf_batched.argtypes = [C.c_int, _f32p, C.c_int64, C.c_int, _i32p, _i32p, _f64p, C.c_int]
        L.oracle_sgetrs_batched.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_int64, C.c_int, _i32p, _f32p,
                                            C.c_int64, C.c_int, C.c_int]
        L.oracle_sgetri_batched.argtypes = [C.c_int, _f32p, C.c_int64, C.c_int, _i32p, _f32p, C.c_int64, C.c_int,
                                            _i32p, C.c_int]
        L.oracle_sgeqrf_batched.argtypes = [C.c_int, C.c_int, _f32p, C.c_int64, C.c_int, _f32p, C.c_int64, C.c_int]
        L.oracle_sgels_batched.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_int64, C.c_int, _f32p,
                                           C.c_int64, C.c_int, _i32p, C.c_int, _f32p]
        L.oracle_cgemm_batched.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                           C.c_float, C.c_float, C.POINTER(_f32p), C.c_int, C.POINTER(_f32p),
                                           C.c_int, C.POINTER(_f32p), C.c_int, C.c_int]
        L.case_matrix_batch.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_int]
        L.case_rhs_batch.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_int]
        _lib = L
    return _lib


def ref():
    """The reference golden library, or None where it was never built."""
    global _ref
    if _ref is None:
        path = _build.REF_LIB
        if not os.path.exists(path):
            path = _build.build_ref()
            if path is None or not os.path.exists(path):
                return None
        L = C.CDLL(path)
        L.ref_available.restype = C.c_int
        L.ref_openblas_config.restype = C.c_char_p
        L.ref_sgetrf_batched.argtypes = [C.c_int, _f32p, C.c_longlong, C.c_int, _i32p, _i32p, C.c_int, C.c_int]
        L.ref_sgetrf_for_solve.argtypes = [C.c_int, _f32p, C.c_longlong, C.c_int, _i32p, _i32p, C.c_int, C.c_int]
        L.ref_sgetrs_batched.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_longlong, C.c_int, _i32p, _f32p,
                                         C.c_longlong, C.c_int, C.c_int, C.c_int]
        L.ref_sgetri_batched.argtypes = [C.c_int, _f32p, C.c_longlong, C.c_int, _i32p, _f32p, C.c_longlong, C.c_int,
                                         _i32p, C.c_int, C.c_int]
        L.ref_sgels_batched.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_longlong, C.c_int, _f32p,
                                        C.c_longlong, C.c_int, _i32p, C.c_int, C.c_int]
        L.ref_sgeqrf_batched.argtypes = [C.c_int, C.c_int, _f32p, C.c_longlong, C.c_int, _f32p, C.c_longlong, _i32p,
                                         C.c_int, C.c_int]
        if not L.ref_available():
            return None
        _ref = L
    return _ref


def _check(a, ncols, ld):
    assert a.dtype == np.float32 and a.flags.c_contiguous and a.ndim == 3, "float32 (batch, ncols, ld) expected"
    assert a.shape[1] >= ncols and a.shape[2] >= ld


# ----------------------------------------------------------------------------- inputs --

def case_matrices(n, lda, mtype, seed, batch):
    """The reference suites' matrix batch (fill.h makeBlasLapackMatrix), shape (batch, n, lda)."""
    a = np.zeros((batch, max(1, n), lda), np.float32)
    lib().case_matrix_batch(_p(a, _f32p), n, lda, MATRIX_TYPES[mtype], seed, batch)
    return a


def case_rhs(n, nrhs, ldb, seed, batch):
    """The getrs suite's right-hand sides (GenerateBMatrix), shape (batch, nrhs, ldb)."""
    b = np.zeros((batch, max(1, nrhs), ldb), np.float32)
    lib().case_rhs_batch(_p(b, _f32p), n, nrhs, ldb, seed, batch)
    return b


# -------------------------------------------------------------------- project restatement --

def port_getrf(a, n, lda, pivot=True):
    """In-place LU of every matrix in ``a``; returns (piv, info, min_gap)."""
    _check(a, n, lda)
    batch = a.shape[0]
    piv = np.zeros((batch, max(1, n)), np.int32) if pivot else None
    info = np.zeros(batch, np.int32)
    gap = np.ones(batch, np.float64)
    lib().oracle_sgetrf_batched(n, _p(a, _f32p), a.shape[1] * a.shape[2], lda, _p(piv, _i32p), _p(info, _i32p),
                                _p(gap, _f64p), batch)
    return piv, info, gap


def port_getrs(trans, lu, n, lda, piv, b, nrhs, ldb):
    """In-place solve op(A) X = B for every matrix; ``trans`` in 'N', 'T', 'C'."""
    _check(lu, n, lda)
    _check(b, nrhs, ldb)
    lib().oracle_sgetrs_batched(TRANS[trans], n, nrhs, _p(lu, _f32p), lu.shape[1] * lu.shape[2], lda,
                                _p(piv, _i32p), _p(b, _f32p), b.shape[1] * b.shape[2], ldb, lu.shape[0])


def port_getri(lu, n, lda, piv, c, ldc):
    """C = inverse from the LU factors; returns info."""
    _check(lu, n, lda)
    _check(c, n, ldc)
    info = np.zeros(lu.shape[0], np.int32)
    lib().oracle_sgetri_batched(n, _p(lu, _f32p), lu.shape[1] * lu.shape[2], lda, _p(piv, _i32p), _p(c, _f32p),
                                c.shape[1] * c.shape[2], ldc, _p(info, _i32p), lu.shape[0])
    return info


def port_geqrf(a, m, n, lda):
    """In-place Householder QR of every matrix of ``a`` (batch, n, lda); returns tau (batch, min(m,n))."""
    _check(a, n, lda)
    k = max(1, min(m, n))
    tau = np.zeros((a.shape[0], k), np.float32)
    lib().oracle_sgeqrf_batched(m, n, _p(a, _f32p), a.shape[1] * a.shape[2], lda, _p(tau, _f32p), k, a.shape[0])
    return tau


def port_gels(trans, a, m, n, nrhs, lda, c, ldc):
    """In place: a (batch, n, lda) factored (transposed first for 'T'), c (batch, nrhs, ldc) the
    solutions; returns info per matrix. trans in 'N', 'T'."""
    _check(a, n, lda)
    _check(c, nrhs, ldc)
    info = np.zeros(a.shape[0], np.int32)
    scratch = np.zeros(max(1, lda * n), np.float32)
    lib().oracle_sgels_batched(1 if trans == "T" else 0, m, n, nrhs, _p(a, _f32p), a.shape[1] * a.shape[2], lda,
                               _p(c, _f32p), c.shape[1] * c.shape[2], ldc, _p(info, _i32p), a.shape[0],
                               _p(scratch, _f32p))
    return info


def _ptr_array(x, batch, skip=()):
    """float* array over the matrices of x (batch, ncols, ld) complex64; None entries at ``skip``."""
    arr = (_f32p * max(1, batch))()
    for b in range(batch):
        if b not in skip:
            arr[b] = x[b].ctypes.data_as(_f32p)
    return arr


def port_cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, skip_c=()):
    """C restatement of aclblasCgemmBatched, in place on c. a, b, c: complex64 arrays
    (batch, ncols, ld); alpha, beta: Python complex; ta, tb in 'N', 'T', 'C'; matrices whose index
    is in ``skip_c`` have a null C pointer."""
    for x in (a, b, c):
        assert x.dtype == np.complex64 and x.flags.c_contiguous and x.ndim == 3
    batch = c.shape[0]
    lib().oracle_cgemm_batched(TRANS[ta], TRANS[tb], m, n, k, alpha.real, alpha.imag, beta.real, beta.imag,
                               _ptr_array(a, batch), lda, _ptr_array(b, batch), ldb,
                               _ptr_array(c, batch, set(skip_c)), ldc, batch)


# ----------------------------------------------------------------- reference golden path --

def ref_cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    """The reference's Cgemm golden (test/gemm_batched/cgemm_batched/cgemm_batched_golden.h:19-64)
    over the BLAS it calls: alpha == 0 scales C by beta in FP32 (ApplyComplexAlphaZeroGolden),
    every other case is cblas_cgemm -- here scipy's OpenBLAS cgemm, the same routine through its
    Fortran interface. In place on c (complex64, (batch, ncols, ld))."""
    from scipy.linalg import blas

    if m == 0 or n == 0:
        return
    trans = {"N": 0, "T": 1, "C": 2}
    br, bi = np.float32(beta.real), np.float32(beta.imag)
    for i in range(c.shape[0]):
        cm = c[i].T[:m, :n]  # column-major m x n view
        if alpha == 0:
            cr, ci = cm.real.copy(), cm.imag.copy()
            cm.real = br * cr - bi * ci
            cm.imag = br * ci + bi * cr
            continue
        ra, ca = (m, k) if ta == "N" else (k, m)
        rb, cb = (k, n) if tb == "N" else (n, k)
        if k == 0:
            # BLAS with k == 0: C = beta C (zero when beta == 0)
            cm[...] = 0 if beta == 0 else (np.complex64(beta) * cm)
            continue
        am = np.asfortranarray(a[i].T[:ra, :ca])
        bm = np.asfortranarray(b[i].T[:rb, :cb])
        out = blas.cgemm(np.complex64(alpha), am, bm, beta=np.complex64(beta), c=np.asfortranarray(cm),
                         trans_a=trans[ta], trans_b=trans[tb])
        cm[...] = out

def ref_getrf(a, n, lda, pivot=True, nthreads=0):
    """aclblasSgetrfBatched_cpu in place; returns (piv, info)."""
    L = ref()
    assert L is not None, "reference golden library unavailable"
    _check(a, n, lda)
    batch = a.shape[0]
    piv = np.zeros((batch, max(1, n)), np.int32) if pivot else None
    info = np.full(batch, -1, np.int32)
    rc = L.ref_sgetrf_batched(n, _p(a, _f32p), a.shape[1] * a.shape[2], lda, _p(piv, _i32p), _p(info, _i32p),
                              batch, nthreads)
    assert rc == 0, rc
    return piv, info


def ref_getrf_for_solve(a, n, lda, pivot=True, nthreads=0):
    """The factorisation the reference's getrs/getri tests prepare (LAPACK, no pivot zeroing)."""
    L = ref()
    assert L is not None, "reference golden library unavailable"
    _check(a, n, lda)
    batch = a.shape[0]
    piv = np.zeros((batch, max(1, n)), np.int32) if pivot else None
    info = np.full(batch, -1, np.int32)
    L.ref_sgetrf_for_solve(n, _p(a, _f32p), a.shape[1] * a.shape[2], lda, _p(piv, _i32p), _p(info, _i32p), batch,
                           nthreads)
    return piv, info


def ref_getrs(trans, lu, n, lda, piv, b, nrhs, ldb, nthreads=0):
    L = ref()
    assert L is not None, "reference golden library unavailable"
    rc = L.ref_sgetrs_batched(TRANS_ACL[trans], n, nrhs, _p(lu, _f32p), lu.shape[1] * lu.shape[2], lda,
                              _p(piv, _i32p), _p(b, _f32p), b.shape[1] * b.shape[2], ldb, lu.shape[0], nthreads)
    assert rc == 0, rc


def ref_geqrf(a, m, n, lda, nthreads=0):
    """aclblasSgeqrfBatched_cpu (LAPACK sgeqrf_) in place; returns tau (batch, min(m,n))."""
    L = ref()
    assert L is not None, "reference golden library unavailable"
    _check(a, n, lda)
    k = max(1, min(m, n))
    tau = np.zeros((a.shape[0], k), np.float32)
    info = np.zeros(1, np.int32)
    rc = L.ref_sgeqrf_batched(m, n, _p(a, _f32p), a.shape[1] * a.shape[2], lda, _p(tau, _f32p), k, _p(info, _i32p),
                              a.shape[0], nthreads)
    assert rc == 0 and info[0] == 0, (rc, info[0])
    return tau


def ref_gels(trans, a, m, n, nrhs, lda, c, ldc, nthreads=0):
    """aclblasSgelsBatched_cpu (LAPACK sgels_) per matrix; c receives the solution rows."""
    L = ref()
    assert L is not None, "reference golden library unavailable"
    info = np.zeros(a.shape[0], np.int32)
    rc = L.ref_sgels_batched(TRANS_ACL[trans], m, n, nrhs, _p(a, _f32p), a.shape[1] * a.shape[2], lda, _p(c, _f32p),
                             c.shape[1] * c.shape[2], ldc, _p(info, _i32p), a.shape[0], nthreads)
    assert rc == 0, rc
    return info


def ref_getri(lu, n, lda, piv, c, ldc, nthreads=0):
    L = ref()
    assert L is not None, "reference golden library unavailable"
    info = np.full(lu.shape[0], -1, np.int32)
    rc = L.ref_sgetri_batched(n, _p(lu, _f32p), lu.shape[1] * lu.shape[2], lda, _p(piv, _i32p), _p(c, _f32p),
                              c.shape[1] * c.shape[2], ldc, _p(info, _i32p), lu.shape[0], nthreads)
    assert rc == 0, rc
    return info


# ---------------------------------------------------------------------------- tolerances --

def ulp_at(x):
    """ULP of |x| in FP32 as the reference verifier defines it (test/frame/verify.h:217-226)."""
    ax = np.abs(np.asarray(x, np.float64))
    e = np.frexp(ax)[1]
    ulp = np.ldexp(1.0, np.maximum(e - 1, -126) - 23)
    return np.where(ax == 0.0, 2.0 ** (-126 - 23), ulp)


def mixed_tolerance_ok(out, gold):
    """The reference's MIXED_TOLERANCE rule for FP32 (test/frame/verify.h:234-333): elements
    equal (or both NaN) are skipped; any NaN/Inf among the rest fails; every element within
    max(1e-2, 32 ulp(|gold|)); at least 99 % within 2^-16 + 2^-10 |gold|."""
    o = np.asarray(out, np.float32).ravel()
    g = np.asarray(gold, np.float32).ravel()
    skip = (o == g) | (np.isnan(o) & np.isnan(g))
    o, g = o[~skip].astype(np.float64), g[~skip].astype(np.float64)
    count = skip.size
    if o.size == 0:
        return True
    if not (np.all(np.isfinite(o)) and np.all(np.isfinite(g))):
        return False
    diff = np.abs(o - g)
    ulp_limit = np.maximum(1e-2, 32.0 * ulp_at(g))
    if np.any(diff > ulp_limit):
        return False
    fails = np.count_nonzero(diff > 1.52587890625e-5 + 0.0009765625 * np.abs(g))
    return (count - fails) / count >= 0.99


def mere_mare_ok(out, gold, threshold=1.0 / 8192.0, multiplier=10.0):
    """The reference's MERE_MARE rule (test/frame/verify.h:153-200): elements equal or both NaN
    are skipped; an Inf among the rest fails; with rel = |out - gold| / (|gold| + 2^-14), the mean
    of rel must stay below ``threshold`` and its maximum below ``multiplier * threshold``."""
    o = np.asarray(out, np.float32).ravel()
    g = np.asarray(gold, np.float32).ravel()
    skip = (o == g) | (np.isnan(o) & np.isnan(g))
    o, g = o[~skip].astype(np.float64), g[~skip].astype(np.float64)
    if o.size == 0:
        return True
    if np.any(np.isinf(o)) or np.any(np.isinf(g)):
        return False
    rel = np.abs(o - g) / (np.abs(g) + 2.0 ** -14)
    return bool(rel.mean() < threshold and rel.max() < multiplier * threshold)


def backward_error(M, x, b):
    """Normwise backward error ||b - M x||_inf / (||M||_inf ||x||_inf + ||b||_inf), in FP64.
    M is the (n, n) matrix in row-major numpy orientation, x and b are (n,) or (n, nrhs)."""
    M = np.asarray(M, np.float64)
    x = np.asarray(x, np.float64)
    b = np.asarray(b, np.float64)
    r = b - M @ x
    den = np.linalg.norm(M, np.inf) * np.abs(x).max() + np.abs(b).max()
    return float(np.abs(r).max() / den) if den > 0 else 0.0


def normwise_rel(out, gold):
    o = np.asarray(out, np.float64)
    g = np.asarray(gold, np.float64)
    den = np.linalg.norm(g)
    return float(np.linalg.norm(o - g) / (den if den > 0 else 1.0))
