"""GPU checks of aclblasSgemmBatched through the C ABI, on every success row of the reference's
sgemm_batched CSV: C = alpha op(A) op(B) + beta C against a float64 product, within the FP32
accumulation bound 2 k u sum|alpha a b| + 2 u |beta c| (u = 2^-24); C outside its m x n block
untouched; k == 0 or alpha == 0 scales C by beta."""
from __future__ import annotations

import zlib

import numpy as np
import pytest

from cases import SGEMM_CASES
from conftest import to_dev, to_host

pytestmark = pytest.mark.gpu
U = 2.0 ** -24


def _op(x, t):
    return x if t == "N" else np.swapaxes(x, 1, 2)


@pytest.mark.parametrize("c", [c for c in SGEMM_CASES if c[3] > 0 and c[4] > 0 and c[11] > 0], ids=lambda c: c[0])
def test_sgemm_batched_csv(handle, c):
    import torch

    name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = c
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    ra, ca = (k, m) if ta != "N" else (m, k)
    rb, cb = (n, k) if tb != "N" else (k, n)
    # column-major storage: array [batch, column, leading dimension]
    a = rng.standard_normal((batch, max(1, ca), lda)).astype(np.float32)
    b = rng.standard_normal((batch, max(1, cb), ldb)).astype(np.float32)
    cm = (rng.standard_normal((batch, n, ldc)) if cfill == "R" else np.zeros((batch, n, ldc))).astype(np.float32)
    cm[:, :, m:] = 77.0
    A = np.swapaxes(a[:, :ca, :ra], 1, 2).astype(np.float64)  # [batch, rows, cols]
    B = np.swapaxes(b[:, :cb, :rb], 1, 2).astype(np.float64)
    C0 = np.swapaxes(cm[:, :, :m], 1, 2).astype(np.float64)
    Cd = to_dev(cm, "cuda")
    handle.sgemm(ta, tb, m, n, k, alpha, to_dev(a, "cuda"), lda, to_dev(b, "cuda"), ldb, beta, Cd, ldc)
    torch.cuda.synchronize()
    out = to_host(Cd)
    assert np.all(out[:, :, m:] == 77.0), "rows beyond m must be untouched"
    got = np.swapaxes(out[:, :, :m], 1, 2).astype(np.float64)
    if k == 0 or alpha == 0.0:
        want = beta * C0 if beta != 1.0 else C0
        np.testing.assert_allclose(got, want, rtol=2 * U, atol=0)
        return
    opa, opb = _op(A, ta), _op(B, tb)
    want = alpha * (opa @ opb) + (beta * C0 if beta != 0.0 else 0.0)
    bound = 2 * k * U * abs(alpha) * (np.abs(opa) @ np.abs(opb)) + 2 * U * abs(beta) * np.abs(C0) + 1e-30
    assert np.all(np.abs(got - want) <= bound + 4 * U * np.abs(want)), name
