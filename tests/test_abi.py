"""C-ABI checks that need no GPU: the library loads, exports every entry point that
include/*.h declares, and applies the reference's host-side validation (status codes, their
order, getrs' -position info) before touching any device state.

Validation failures and the n == 0 / batch == 0 no-op paths return before the handle is
dereferenced (as in sgetrf_batched_host.cpp:66-84), so these tests pass a non-null dummy
handle and dummy non-null pointers, which are never read.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import re

import pytest

from cases import (CGEMM_ERRORS, GELS_ROWS, GEQRF_ROWS, GETRF_ERRORS, GETRI_ERRORS, GETRS_ERRORS, MATINV_ARG_ROWS,
                   SGEMM_ERRORS)
from conftest import ROOT

DUMMY = C.create_string_buffer(256)
H = C.cast(DUMMY, C.c_void_p)
P = C.c_void_p(0x1000)  # non-null, never dereferenced on these paths


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names += re.findall(r"^\s*(?:ACLBLAS_EXPORT\s+)?aclblasStatus_t\s+(aclblas\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(ob):
    lib = ob.lib()
    names = declared_symbols()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(names) == set(ob.SIGNATURES), "the Python binding must cover exactly the declared API"


def test_status_and_operation_values_match_reference(ob):
    text = open(os.path.join(ROOT, "include", "cann_ops_blas_common.h")).read()
    vals = dict(re.findall(r"ACLBLAS_STATUS_(\w+)\s*=\s*(\d+)", text))
    for code, name in ob.STATUS.items():
        assert int(vals[name]) == code
    assert (ob.OP_N, ob.OP_T, ob.OP_C) == (111, 112, 113)


def test_version(ob):
    v = C.c_int(0)
    assert ob.lib().aclblasGetVersion(None, C.byref(v)) == ob.SUCCESS
    assert v.value == 10000
    assert ob.lib().aclblasGetVersion(None, None) == ob.INVALID_VALUE


def test_handle_argument_checks(ob):
    L = ob.lib()
    assert L.aclblasCreate(None) == ob.HANDLE_IS_NULLPTR
    h = C.c_void_p(0x10)
    assert L.aclblasCreate(C.byref(h)) == ob.INVALID_VALUE  # *handle must be NULL
    assert L.aclblasDestroy(None) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSetStream(None, None) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasGetStream(None, None) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasGetStream(H, None) == ob.INVALID_VALUE
    assert L.aclblasSetWorkspace(None, P, 16) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSetWorkspace(H, None, 16) == ob.INVALID_VALUE
    assert L.aclblasSetWorkspace(H, P, 0) == ob.INVALID_VALUE


def test_create_without_device_fails_cleanly(ob):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    st = ob.lib().aclblasCreate(C.byref(h))
    assert st in (ob.NOT_INITIALIZED, ob.ALLOC_FAILED)
    assert not h.value


@pytest.mark.parametrize("row", GETRF_ERRORS, ids=lambda r: r[0])
def test_getrf_error_rows(ob, row):
    name, n, lda, batch, null_a, null_info, null_h, status = row
    st = ob.lib().aclblasSgetrfBatched(None if null_h else H, n, None if null_a else P, lda, P,
                                       None if null_info else P, batch)
    assert ob.STATUS[st] == status


def test_getrf_validation_order(ob):
    L = ob.lib()
    # lda is checked before the n == 0 no-op (sgetrf_batched_host.cpp:43-52)
    assert L.aclblasSgetrfBatched(H, 0, None, 0, None, None, 4) == ob.INVALID_VALUE
    assert L.aclblasSgetrfBatched(H, 0, None, 1, None, None, 4) == ob.SUCCESS
    assert L.aclblasSgetrfBatched(H, 8, None, 8, None, None, 0) == ob.SUCCESS
    # no-pivot mode may omit infoArray; pivot mode may not
    assert L.aclblasSgetrfBatched(H, 8, None, 8, None, None, 2) == ob.INVALID_VALUE  # Aarray NULL
    assert L.aclblasSgetrfBatched(H, 8, P, 8, P, None, 2) == ob.INVALID_VALUE
    assert L.aclblasSgetrfBatched(None, -1, None, 0, None, None, -1) == ob.HANDLE_IS_NULLPTR


@pytest.mark.parametrize("row", GETRS_ERRORS, ids=lambda r: r[0])
def test_getrs_error_rows(ob, row):
    name, trans, n, nrhs, lda, ldb, batch, null_a, null_b, null_h, status, exp_info = row
    info = C.c_int(12345)
    t = 999 if trans == "INVALID" else ob.TRANS[trans]
    st = ob.lib().aclblasSgetrsBatched(None if null_h else H, t, n, nrhs, None if null_a else P, lda, P,
                                       None if null_b else P, ldb, C.byref(info), batch)
    assert ob.STATUS[st] == status
    if exp_info is None:
        assert info.value == 12345  # handle errors leave info untouched
    else:
        assert info.value == exp_info


def test_getrs_info_and_noop(ob):
    L = ob.lib()
    info = C.c_int(-99)
    # valid no-op calls set *info = 0 (sgetrs_batched_host.cpp:178-182) without touching arrays
    assert L.aclblasSgetrsBatched(H, ob.OP_N, 0, 4, None, 1, None, None, 1, C.byref(info), 4) == ob.SUCCESS
    assert info.value == 0
    info.value = -99
    assert L.aclblasSgetrsBatched(H, ob.OP_T, 32, 0, None, 32, None, None, 32, C.byref(info), 4) == ob.SUCCESS
    assert info.value == 0
    # info may be NULL
    assert L.aclblasSgetrsBatched(H, ob.OP_N, 32, 4, None, 32, None, P, 32, None, 4) == ob.INVALID_VALUE
    # position precedence: trans beats n
    info.value = 0
    assert L.aclblasSgetrsBatched(H, 0, -1, -1, None, 0, None, None, 0, C.byref(info), -1) == ob.INVALID_ENUM
    assert info.value == -2


@pytest.mark.parametrize("row", GETRI_ERRORS, ids=lambda r: r[0])
def test_getri_error_rows(ob, row):
    name, n, lda, ldc, batch, null_a, null_c, null_info, null_h, status = row
    st = ob.lib().aclblasSgetriBatched(None if null_h else H, n, None if null_a else P, lda, P,
                                       None if null_c else P, ldc, None if null_info else P, batch)
    assert ob.STATUS[st] == status


def test_getri_noop_and_null_handle(ob):
    L = ob.lib()
    assert L.aclblasSgetriBatched(None, 32, None, 32, None, None, 32, None, 4) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSgetriBatched(H, 0, None, 1, None, None, 1, None, 4) == ob.SUCCESS
    assert L.aclblasSgetriBatched(H, 32, None, 32, None, None, 32, None, 0) == ob.SUCCESS


@pytest.mark.parametrize("row", MATINV_ARG_ROWS, ids=lambda r: r[0])
def test_matinv_argument_rows(ob, row):
    name, n, lda, lda_inv, batch, null_a, null_ainv, null_info, status = row
    st = ob.lib().aclblasSmatinvBatched(H, n, None if null_a else P, lda, None if null_ainv else P, lda_inv,
                                        None if null_info else P, batch)
    assert ob.STATUS[st] == status


def test_matinv_null_handle(ob):
    assert ob.lib().aclblasSmatinvBatched(None, -1, None, 0, None, 0, None, -1) == ob.HANDLE_IS_NULLPTR


@pytest.mark.parametrize("row", SGEMM_ERRORS, ids=lambda r: r[0])
def test_sgemm_batched_error_rows(ob, row):
    name, ta, tb, m, n, k, lda, ldb, ldc, batch, nulls, null_h, status = row
    one = C.c_float(1.0)
    op = lambda t: 999 if t == "INVALID" else ob.TRANS[t]
    ptr = lambda null, p: None if null else p
    st = ob.lib().aclblasSgemmBatched(None if null_h else H, op(ta), op(tb), m, n, k, ptr(nulls[0], C.byref(one)),
                                      ptr(nulls[2], P), lda, ptr(nulls[3], P), ldb, ptr(nulls[1], C.byref(one)),
                                      ptr(nulls[4], P), ldc, batch)
    assert ob.STATUS[st] == status


def test_sgemm_batched_noops(ob):
    L, one = ob.lib(), C.c_float(1.0)
    # m, n or batch zero: success before any array is read (gemm_batched_host.cpp:420-422)
    assert L.aclblasSgemmBatched(H, ob.OP_N, ob.OP_N, 0, 128, 128, C.byref(one), P, 1, P, 128, C.byref(one), P, 1,
                                 4) == ob.SUCCESS
    assert L.aclblasSgemmBatched(H, ob.OP_N, ob.OP_N, 8, 8, 8, C.byref(one), None, 8, None, 8, C.byref(one), None, 8,
                                 0) == ob.SUCCESS
    # k == 0 with beta == 1 leaves C untouched without a launch
    assert L.aclblasSgemmBatched(H, ob.OP_N, ob.OP_N, 8, 8, 0, C.byref(one), P, 8, P, 1, C.byref(one), P, 8,
                                 4) == ob.SUCCESS


@pytest.mark.parametrize("row", CGEMM_ERRORS, ids=lambda r: r[0])
def test_cgemm_batched_error_rows(ob, row):
    name, ta, tb, m, n, k, lda, ldb, ldc, batch, nulls, null_h, status = row
    one = (C.c_float * 2)(1.0, 0.0)
    op = lambda t: 999 if t == "INVALID" else ob.TRANS[t]
    ptr = lambda null, p: None if null else p
    st = ob.lib().aclblasCgemmBatched(None if null_h else H, op(ta), op(tb), m, n, k, ptr(nulls[0], one),
                                      ptr(nulls[2], P), lda, ptr(nulls[3], P), ldb, ptr(nulls[1], one),
                                      ptr(nulls[4], P), ldc, batch)
    assert ob.STATUS[st] == status


def test_cgemm_batched_validation_order_and_noops(ob):
    L = ob.lib()
    one = (C.c_float * 2)(1.0, 0.0)
    zero = (C.c_float * 2)(0.0, 0.0)
    # alpha is checked before the dimensions, the operations before the leading dimensions
    assert L.aclblasCgemmBatched(H, ob.OP_N, ob.OP_N, -1, 8, 8, None, P, 8, P, 8, one, P, 8, 1) == ob.INVALID_VALUE
    assert L.aclblasCgemmBatched(H, 999, ob.OP_N, 8, 8, 8, one, P, 1, P, 8, one, P, 8, 1) == ob.INVALID_VALUE
    # conjugate transpose takes its leading dimension from k, like T
    assert L.aclblasCgemmBatched(H, ob.OP_C, ob.OP_N, 128, 8, 16, one, P, 15, P, 16, one, P, 128,
                                 1) == ob.INVALID_VALUE
    # m, n or batch zero: success before any array is read (gemm_batched_host.cpp:791-793)
    assert L.aclblasCgemmBatched(H, ob.OP_N, ob.OP_N, 0, 128, 128, one, P, 1, P, 128, one, P, 1, 4) == ob.SUCCESS
    assert L.aclblasCgemmBatched(H, ob.OP_N, ob.OP_N, 8, 8, 8, one, None, 8, None, 8, one, None, 8, 0) == ob.SUCCESS
    # k == 0 or alpha == 0 with beta == 1 leaves C untouched without a launch (:801-804)
    assert L.aclblasCgemmBatched(H, ob.OP_N, ob.OP_N, 8, 8, 0, one, P, 8, P, 1, one, P, 8, 4) == ob.SUCCESS
    assert L.aclblasCgemmBatched(H, ob.OP_T, ob.OP_C, 8, 8, 8, zero, P, 8, P, 8, one, P, 8, 4) == ob.SUCCESS


def _geqrf_expected_info(m, n, lda, batch, null_a, null_tau):
    """LAPACK-style -position of ValidateGeqrfBatchedParams (sgeqrf_batched_host.cpp:21-58)."""
    if m < 0:
        return -1
    if n < 0:
        return -2
    if lda < max(1, m):
        return -4
    if batch < 0:
        return -6
    if batch > 0 and null_a:
        return -3
    if batch > 0 and m > 0 and n > 0 and null_tau:
        return -5
    return 0


@pytest.mark.parametrize("row", [r for r in GEQRF_ROWS if r[8] != "SUCCESS" or min(r[1], r[2], r[4]) == 0],
                         ids=lambda r: r[0])
def test_geqrf_argument_rows(ob, row):
    name, m, n, lda, batch, fill, null_a, null_tau, status = row
    info = C.c_int(12345)
    st = ob.lib().aclblasSgeqrfBatched(H, m, n, None if null_a else P, lda, None if null_tau else P, C.byref(info),
                                       batch)
    assert ob.STATUS[st] == status
    assert info.value == _geqrf_expected_info(m, n, lda, batch, null_a, null_tau)


def test_geqrf_null_handle_and_info(ob):
    L, info = ob.lib(), C.c_int(7)
    assert L.aclblasSgeqrfBatched(None, 8, 8, P, 8, P, C.byref(info), 2) == ob.HANDLE_IS_NULLPTR
    assert info.value == 7
    assert L.aclblasSgeqrfBatched(H, 8, 8, P, 8, P, None, 2) == ob.INVALID_VALUE


@pytest.mark.parametrize("row", [r for r in GELS_ROWS if r[10] != "SUCCESS" or min(r[2], r[3], r[4], r[7]) == 0],
                         ids=lambda r: r[0])
def test_gels_argument_rows(ob, row):
    name, t, m, n, nrhs, lda, ldc, batch, cfill, null, status, desc = row
    op = 999 if t == "X" else ob.TRANS[t]
    st = ob.lib().aclblasSgelsBatched(None if null == "H" else H, op, m, n, nrhs, None if null == "A" else P, lda,
                                      None if null == "C" else P, ldc, None if null == "I" else P, batch)
    assert ob.STATUS[st] == status


def test_strided_and_builder_validation(ob):
    L, info = ob.lib(), C.c_int(0)
    assert L.aclblasBuildPointerArray(None, P, 16, 4, P) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasBuildPointerArray(H, P, 16, -1, P) == ob.INVALID_VALUE
    assert L.aclblasBuildPointerArray(H, None, 16, 4, P) == ob.INVALID_VALUE
    assert L.aclblasBuildPointerArray(H, None, 16, 0, None) == ob.SUCCESS
    # the batched calls' validation and no-op paths, reached before any pointer array is built
    assert L.aclblasSgetrfStridedBatched(None, 8, P, 8, 64, P, P, 2) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSgetrfStridedBatched(H, -1, P, 8, 64, P, P, 2) == ob.INVALID_VALUE
    assert L.aclblasSgetrfStridedBatched(H, 0, P, 1, 0, P, P, 2) == ob.SUCCESS
    assert L.aclblasSgetrfStridedBatched(H, 8, None, 8, 64, P, P, 2) == ob.INVALID_VALUE
    assert L.aclblasSgetrsStridedBatched(H, 999, 8, 1, P, 8, 64, P, P, 8, 8, C.byref(info), 2) == ob.INVALID_ENUM
    assert L.aclblasSgetrsStridedBatched(H, ob.OP_N, 8, 0, P, 8, 64, P, P, 8, 8, C.byref(info), 2) == ob.SUCCESS
    assert L.aclblasSgetriStridedBatched(H, 8, P, 8, 64, P, None, 8, 64, P, 2) == ob.INVALID_VALUE
    assert L.aclblasSgetriStridedBatched(H, 8, P, 8, 64, P, P, 8, 64, P, 0) == ob.SUCCESS


def test_logger_callback_receives_validation_errors(ob):
    L = ob.lib()
    seen = []
    cb_t = C.CFUNCTYPE(None, C.c_char_p)
    cb = cb_t(lambda msg: seen.append(msg.decode()))
    assert L.aclblasSetLoggerCallback(C.cast(cb, C.c_void_p)) == ob.SUCCESS
    got = C.c_void_p()
    assert L.aclblasGetLoggerCallback(C.byref(got)) == ob.SUCCESS
    assert got.value == C.cast(cb, C.c_void_p).value
    try:
        assert L.aclblasSgetrfBatched(H, -3, P, 1, P, P, 1) == ob.INVALID_VALUE
    finally:
        L.aclblasSetLoggerCallback(None)
    assert any("aclblasSgetrfBatched" in s and "n must be >= 0" in s for s in seen)
    assert L.aclblasGetLoggerCallback(None) == ob.INVALID_VALUE
    assert L.aclblasLoggerConfigure(0, 0, 0, None) == ob.SUCCESS


def test_logger_file_sink(ob, tmp_path):
    L = ob.lib()
    path = str(tmp_path / "log.txt").encode()
    buf = C.create_string_buffer(path)
    assert L.aclblasLoggerConfigure(1, 0, 0, buf) == ob.SUCCESS
    try:
        L.aclblasSgetriBatched(H, 5, P, 3, P, P, 5, P, 4)
    finally:
        L.aclblasLoggerConfigure(0, 0, 0, None)
    text = open(path.decode()).read()
    assert "lda must be >= max(1, n)" in text


from cases import GEMM_ERRORS  # noqa: E402

DT = {"F32": 0, "F16": 1, "BF16": 27, "E5M2": 35, "E4M3": 36}
CT = {"16F": 0, "32F": 2}


@pytest.mark.parametrize("row", GEMM_ERRORS, ids=lambda r: r[0])
def test_gemm_batched_ex_error_rows(ob, row):
    (name, ta, tb, m, n, k, at, bt, ct, lda, ldb, ldc, batch, comp, algo, an, bn, a0, b0, c0, hn, status) = row
    one = C.c_float(1.0)
    zero = C.c_float(0.0)
    tr = lambda t: 999 if t == "INVALID" else ob.TRANS[t]  # noqa: E731
    st = ob.lib().aclblasGemmBatchedEx(
        None if hn else H, tr(ta), tr(tb), m, n, k, None if an else C.byref(one), None if a0 else P, DT[at], lda,
        None if b0 else P, DT[bt], ldb, None if bn else C.byref(zero), None if c0 else P, DT[ct], ldc, batch,
        CT[comp], algo)
    assert ob.STATUS[st] == status


def test_gemm_batched_ex_fp32_extension_and_noop(ob):
    L = ob.lib()
    one, zero = C.c_float(1.0), C.c_float(0.0)
    # FP32 operands accepted with the PEDANTIC and FAST compute types (no-op sizes: nothing touched)
    for comp in (3, 5, 6):
        assert L.aclblasGemmBatchedEx(H, ob.OP_N, ob.OP_N, 0, 4, 4, C.byref(one), P, 0, 4, P, 0, 4, C.byref(zero),
                                      P, 0, 4, 2, comp, 0) == ob.SUCCESS
    assert L.aclblasGemmBatchedEx(H, ob.OP_N, ob.OP_N, 4, 4, 4, C.byref(one), P, 0, 4, P, 0, 4, C.byref(zero), P,
                                  0, 4, 0, 6, 0) == ob.SUCCESS


def test_refine_and_adjoint_validation(ob):
    L = ob.lib()
    assert L.aclblasSgetrfsRefineBatchedEx(None, 4, 1, P, 4, P, 4, P, P, 4, P, 4, 6, 5, 1e-6, P, P, P, 2) == \
        ob.HANDLE_IS_NULLPTR
    assert L.aclblasSgetrfsRefineBatchedEx(H, 4, 1, P, 3, P, 4, P, P, 4, P, 4, 6, 5, 1e-6, P, P, P, 2) == \
        ob.INVALID_VALUE
    assert L.aclblasSgetrfsRefineBatchedEx(H, 4, 1, P, 4, P, 4, P, P, 4, P, 4, 0, 5, 1e-6, P, P, P, 2) == \
        ob.NOT_SUPPORTED
    assert L.aclblasSgetrfsRefineBatchedEx(H, 0, 1, None, 1, None, 1, None, None, 1, None, 1, 6, 5, 1e-6, None,
                                           None, None, 2) == ob.SUCCESS
    assert L.aclblasSgetrsAdjointBatched(None, 4, 1, P, 4, P, P, 4, P, 4, P, 4, 2) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSgetrsAdjointBatched(H, 4, 257, P, 4, P, P, 4, P, 4, P, 4, 2) == ob.INVALID_VALUE
    assert L.aclblasSgetrsAdjointBatched(H, 4, 2, P, 4, P, P, 3, P, 4, P, 4, 2) == ob.INVALID_VALUE
    assert L.aclblasSgetrsAdjointBatched(H, 4, 0, None, 4, None, None, 4, None, 4, None, 4, 2) == ob.SUCCESS


def test_grouped_argument_checks(ob):
    """Plan creation validates every group before touching the device."""
    L = ob.lib()
    ia = ob._int_array
    plan = C.c_void_p()
    args = lambda ns, nrhs, lda, ldb, sz: (len(ns), ia(ns), ia(nrhs), ia(lda), ia(ldb), ia(sz), None, C.byref(plan))
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(None, *args([4], [1], [4], [4], [2])) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, *args([-1], [1], [4], [4], [2])) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, *args([4], [-1], [4], [4], [2])) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, *args([4], [1], [3], [4], [2])) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, *args([4], [1], [4], [3], [2])) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, *args([4], [1], [4], [4], [-2])) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, 1, None, None, None, None, None, None,
                                                 C.byref(plan)) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, -1, None, None, None, None, None, None,
                                                 C.byref(plan)) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanCreate(H, 0, None, None, None, None, None, None, None) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanDestroy(None) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedPlanGetConfig(None, None) == ob.INVALID_VALUE
    assert L.aclblasSgetrfGetrsGroupedBatched(None, None, P, P, P, P) == ob.HANDLE_IS_NULLPTR
    assert L.aclblasSgetrfGetrsGroupedBatched(H, None, P, P, P, P) == ob.INVALID_VALUE
