"""aclblasSgelsBatched semantics pinned on the CPU: the oracle's restatement of the reference
kernel (oracle/lu_oracle.c) against the reference's golden (LAPACK sgels_ through
test/gels_batched/sgels_batched/sgels_batched_golden.h) on every success row of the reference's
gels CSV: info equal, the solution rows under the suite's MERE_MARE rule (threshold 2^-13,
multiplier 10). The rank-deficient row (a repeated column: the solution is not unique and both
solvers return huge, different components) is compared on info and on the residual instead.
Where MERE_MARE fails on a well-posed row, the two FP32 solvers may still differ by their
conditioning: such a solution passes when its normwise difference is within
max(1e-5, 8 kappa_2(op(A)) 2^-24), the bound two backward-stable solvers can promise."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import GELS_ROWS, gels_inputs

WORK = [r for r in GELS_ROWS if r[10] == "SUCCESS" and min(r[2], r[3], r[4], r[7]) > 0]


@pytest.mark.parametrize("row", WORK, ids=lambda r: r[0])
def test_oracle_gels_matches_reference_golden(row):
    if O.ref() is None:
        pytest.skip("reference golden library unavailable")
    name, t, m, n, nrhs, lda, ldc, batch, cfill, null, status, desc = row
    a, c = gels_inputs(row, 11)
    a1, c1 = a.copy(), c.copy()
    i1 = O.port_gels(t, a1, m, n, nrhs, lda, c1, ldc)
    a2, c2 = a.copy(), c.copy()
    i2 = O.ref_gels(t, a2, m, n, nrhs, lda, c2, ldc)
    np.testing.assert_array_equal(i1, i2)
    sol = n if t == "N" else m
    for b in range(batch):
        if desc == "rank_deficient":
            A = a[b, :n, :m].T.astype(np.float64)
            op = A if t == "N" else A.T
            rows = op.shape[0]
            B = c[b, :, :rows].T.astype(np.float64)
            for x in (c1, c2):
                X = x[b, :, :sol].T.astype(np.float64)
                res = np.linalg.norm(op @ X - B) / (np.linalg.norm(op) * np.linalg.norm(X) + np.linalg.norm(B))
                assert res < 1e-5, (name, b, res)
        elif not O.mere_mare_ok(c1[b, :, :sol], c2[b, :, :sol], 0.0001220703125, 10.0):
            A = a[b, :n, :m].T.astype(np.float64)
            kappa = np.linalg.cond(A)
            rel = O.normwise_rel(c1[b, :, :sol], c2[b, :, :sol])
            assert rel <= max(1e-5, 8.0 * kappa * 2.0 ** -24), (name, b, rel, kappa)
