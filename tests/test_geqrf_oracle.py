"""aclblasSgeqrfBatched semantics pinned on the CPU: the oracle's restatement of the reference
kernel (oracle/lu_oracle.c) against the reference's golden (LAPACK sgeqrf_ through
test/geqrf_batched/sgeqrf_batched/sgeqrf_batched_golden.h) on every success row of the
reference's geqrf CSV, under the reference's own rule for that suite: MERE_MARE on A (R and the
reflectors, padding included) and on tau, with the row's threshold and multiplier; and a
reconstruction check Q R = A in float64.

Two backward-stable QRs (LAPACK scales its norms and multiplies by a reciprocal, the restatement
sums in row order and divides) can differ by a few ulp of ||A|| on an entry that cancels to near
the rule's 2^-14 floor, where the MARE term reads that as a large relative error. Such a matrix
passes when the MERE term holds and every element is within 64 u ||A||_F (u = 2^-24) -- the
normwise statement the MARE term stands in for."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import GEQRF_MARE_MULTIPLIER, GEQRF_ROWS, geqrf_matrices

WORK = [r for r in GEQRF_ROWS if r[8] == "SUCCESS" and min(r[1], r[2], r[4]) > 0]


def qr_reconstruct(a, tau, m, n):
    """Q R of one factored matrix (column-major storage a[col][row]) in float64."""
    A = a[:n, :m].T.astype(np.float64)
    k = min(m, n)
    R = np.triu(A[:k, :])
    Q = np.eye(m)
    for i in reversed(range(k)):
        v = np.zeros(m)
        v[i] = 1.0
        v[i + 1:] = A[i + 1:, i]
        Q = Q - tau[i] * np.outer(v, v @ Q)
    return Q[:, :k] @ R


def parity_ok(out, gold, a, mult):
    if O.mere_mare_ok(out, gold, 0.000122, mult):
        return True
    if not O.mere_mare_ok(out, gold, 0.000122, float("inf")):
        return False
    floor = 64 * 2.0 ** -24 * np.linalg.norm(a.astype(np.float64))
    return bool(np.all(np.abs(out.astype(np.float64) - gold.astype(np.float64)) <= floor))


@pytest.mark.parametrize("row", WORK, ids=lambda r: r[0])
def test_oracle_geqrf_matches_reference_golden(row):
    if O.ref() is None:
        pytest.skip("reference golden library unavailable")
    name, m, n, lda, batch, fill = row[:6]
    a = geqrf_matrices(m, n, lda, fill, 7, batch)
    x = a.copy()
    t = O.port_geqrf(x, m, n, lda)
    g = a.copy()
    tg = O.ref_geqrf(g, m, n, lda)
    mult = GEQRF_MARE_MULTIPLIER.get(name, 10.0)
    for b in range(batch):
        assert parity_ok(x[b], g[b], a[b, :n, :m], mult), (name, b, "A")
        assert parity_ok(t[b], tg[b], a[b, :n, :m], mult), (name, b, "tau")
        assert np.all(x[b, :, m:] == 99.0)
        if fill != "VALUE_NORM_0":
            ref = a[b, :n, :m].T.astype(np.float64)
            err = np.linalg.norm(qr_reconstruct(x[b], t[b], m, n) - ref) / max(np.linalg.norm(ref), 1e-30)
            assert err < 1e-5, (name, b, err)
