"""aclblasSmatinvBatched semantics pinned on the CPU.

The oracle's composition (port_getrf on a copy of A, then port_getri -- the reference's device
sequence of matinv_batched_host.cpp:164-194) is checked against the reference's own matinv golden
rule (test/matinv_batched/matinv_batched_golden.h: LAPACK sgetrf_ on the copy, info from it when
singular, else sgetri_'s): info exact for every row of the reference's matinv CSV, the inverse
under the reference's MIXED_TOLERANCE rule where the CSV compares values (its singular and
ill-conditioned rows compare info only).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import MATINV_CASES, MATINV_SEED


def oracle_matinv(a, n, lda, lda_inv):
    """Ainv (batch, n, lda_inv; -7 outside the n x n block) and info of the device sequence."""
    lu = a.copy()
    piv, _, _ = O.port_getrf(lu, n, lda)
    c = np.full((a.shape[0], n, lda_inv), -7.0, np.float32)
    info = O.port_getri(lu, n, lda, piv, c, lda_inv)
    return c, info


VALUE_ROWS = {"SINGULAR_ZERO_COL", "SINGULAR_DEPENDENT_ROW", "ILL_CONDITIONED"}  # info only in the CSV


@pytest.mark.parametrize("c", MATINV_CASES, ids=lambda c: c[0])
def test_oracle_matinv_matches_reference_golden(c):
    if O.ref() is None:
        pytest.skip("reference golden library unavailable")
    name, n, lda, lda_inv, batch, mtype = c
    a = O.case_matrices(n, lda, mtype, MATINV_SEED, batch)
    oc, oinfo = oracle_matinv(a, n, lda, lda_inv)
    g = a.copy()
    gpiv, ginfo = O.ref_getrf_for_solve(g, n, lda)
    gc = np.full((batch, n, lda_inv), -7.0, np.float32)
    ginfo2 = O.ref_getri(g, n, lda, gpiv, gc, lda_inv)
    gold_info = np.where(ginfo > 0, ginfo, ginfo2)
    np.testing.assert_array_equal(oinfo, gold_info)
    if mtype not in VALUE_ROWS:
        for k in range(batch):
            if gold_info[k] == 0:
                assert O.mixed_tolerance_ok(oc[k, :, :n], gc[k, :, :n]), (name, k)
