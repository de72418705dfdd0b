"""aclblasCgemmBatched semantics pinned on the CPU.

The oracle (port_cgemm: the reference's four real sums and its combine order,
gemm_batched_host.cpp:438-819 and gemm_batched_kernel.cpp:1029-1110) is checked against the
reference's golden (test/gemm_batched/cgemm_batched/cgemm_batched_golden.h: cblas_cgemm, or the
FP32 beta scaling when alpha == 0) on every success row of the reference's Cgemm CSV, under the
reference's own rule: real and imaginary parts each within MIXED_TOLERANCE
(cgemm_batched_test.cpp:118-131). Rows of C beyond m stay untouched.
"""
from __future__ import annotations

import zlib

import numpy as np
import pytest

import oracle as O
from cases import CGEMM_CASES

PAD = np.complex64(77 + 77j)


def cgemm_inputs(c):
    """Seeded inputs of a CSV row: A, B, C as complex64 (batch, ncols, ld) with normal real and
    imaginary parts; C zero or random per the row's c_fill, PAD beyond row m."""
    name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = c
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    ca = k if ta == "N" else m
    cb = n if tb == "N" else k

    def cnormal(shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)

    a = cnormal((batch, max(1, ca), lda))
    b = cnormal((batch, max(1, cb), ldb))
    cm = cnormal((batch, max(1, n), ldc)) if cfill == "R" else np.zeros((batch, max(1, n), ldc), np.complex64)
    cm[:, :, m:] = PAD
    return a, b, cm


VALUE_ROWS = [c for c in CGEMM_CASES if c[3] > 0 and c[4] > 0 and c[11] > 0]


@pytest.mark.parametrize("c", VALUE_ROWS, ids=lambda c: c[0])
def test_oracle_cgemm_matches_reference_golden(c):
    pytest.importorskip("scipy")
    name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = c
    a, b, cm = cgemm_inputs(c)
    out = cm.copy()
    O.port_cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, out, ldc)
    gold = cm.copy()
    O.ref_cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, gold, ldc)
    assert np.all(out[:, :, m:] == PAD), "rows beyond m must be untouched"
    for i in range(batch):
        o, g = out[i, :n, :m], gold[i, :n, :m]
        assert O.mixed_tolerance_ok(o.real, g.real), (name, i, "real")
        assert O.mixed_tolerance_ok(o.imag, g.imag), (name, i, "imag")


def test_oracle_cgemm_noops_and_null_c():
    """m, n or batch zero and (alpha == 0 or k == 0) with beta == 1 write nothing; a null C
    pointer skips its matrix."""
    c = ("x", "N", "N", 5, 4, 3, 1 + 0j, 0j, 5, 3, 5, 2, "R")
    a, b, cm = cgemm_inputs(c)
    for args in ((0, 4, 3, 1 + 0j, 0j), (5, 0, 3, 1 + 0j, 0j), (5, 4, 3, 0j, 1 + 0j), (5, 4, 0, 2 + 1j, 1 + 0j)):
        out = cm.copy()
        m, n, k, al, be = args
        O.port_cgemm("N", "N", m, n, k, al, a, 5, b, 3, be, out, 5)
        assert np.array_equal(out, cm), args
    out = cm.copy()
    O.port_cgemm("N", "N", 5, 4, 3, 1 + 0j, a, 5, b, 3, 0j, out, 5, skip_c=(0,))
    assert np.array_equal(out[0], cm[0]) and not np.array_equal(out[1], cm[1])


def test_oracle_cgemm_alpha_zero_ignores_operands():
    """alpha == 0 combines zero sums: NaN in A or B never reaches C; beta == 0 overwrites NaN in C."""
    c = ("y", "N", "N", 6, 5, 4, 1 + 0j, 0j, 6, 4, 6, 1, "R")
    a, b, cm = cgemm_inputs(c)
    a[:] = np.nan
    out = cm.copy()
    O.port_cgemm("N", "N", 6, 5, 4, 0j, a, 6, b, 4, 0.5 - 0.25j, out, 6)
    assert np.all(np.isfinite(out[:, :, :6]))
    cm[0, 0, 0] = np.nan
    out = cm.copy()
    O.port_cgemm("N", "N", 6, 5, 4, 0j, a, 6, b, 4, 0j, out, 6)
    assert np.all(out[:, :, :6] == 0)
