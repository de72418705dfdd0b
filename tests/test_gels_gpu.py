"""GPU parity of aclblasSgelsBatched through the C ABI: bit for bit against the oracle's
restatement (pinned to the reference's LAPACK golden in test_gels_oracle.py) -- factors, solution
block including the rows the algorithm leaves, padding, and per-matrix info -- on every success
row of the reference's gels CSV, on singular members (a zero column / zero row that stops the
triangular solve), and on a larger batch."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import GELS_ROWS, gels_inputs
from conftest import to_dev, to_host
from test_lu_gpu import assert_bitwise

pytestmark = pytest.mark.gpu


def gpu_gels(handle, t, a, m, n, nrhs, lda, c, ldc):
    import torch

    A, Cd = to_dev(a, "cuda"), to_dev(c, "cuda")
    info = handle.gels(t, A, m, n, nrhs, lda, Cd, ldc)
    torch.cuda.synchronize()
    return to_host(A), to_host(Cd), to_host(info)


def check(handle, t, a, c, m, n, nrhs, lda, ldc, what):
    ga, gc, gi = gpu_gels(handle, t, a, m, n, nrhs, lda, c, ldc)
    oa, oc = a.copy(), c.copy()
    oi = O.port_gels(t, oa, m, n, nrhs, lda, oc, ldc)
    np.testing.assert_array_equal(gi, oi)
    assert_bitwise(ga, oa, what + " A")
    assert_bitwise(gc, oc, what + " C")
    return gi


@pytest.mark.parametrize("row", [r for r in GELS_ROWS if r[10] == "SUCCESS" and min(r[2], r[3], r[4], r[7]) > 0],
                         ids=lambda r: r[0])
def test_gels_csv(handle, row):
    name, t, m, n, nrhs, lda, ldc, batch = row[:8]
    a, c = gels_inputs(row, 11)
    check(handle, t, a, c, m, n, nrhs, lda, ldc, name)


@pytest.mark.parametrize("shape", [("N", 12, 6, 3), ("N", 6, 12, 3), ("T", 12, 6, 2), ("T", 6, 12, 2)])
def test_gels_singular_members(handle, shape):
    t, m, n, nrhs = shape
    lda, ldc, batch = m + 1, max(m, n) + 2, 6
    rng = np.random.default_rng(m * 31 + n)
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    c = rng.standard_normal((batch, nrhs, ldc)).astype(np.float32)
    a[1] = 0.0                   # all zero: every reflector skipped, zero diagonal
    a[2, :, 2] = 0.0             # a zero row of A
    a[3, 1, :] = 0.0             # a zero column of A
    info = check(handle, t, a, c, m, n, nrhs, lda, ldc, f"{t} {m}x{n}")
    assert info[1] > 0


@pytest.mark.parametrize("shape", [("N", 32, 16, 2), ("N", 32, 31, 1), ("N", 20, 3, 29), ("T", 9, 24, 8),
                                   ("T", 1, 32, 3), ("N", 32, 1, 31), ("T", 16, 16, 16)])
def test_gels_warp_path_shapes(handle, shape):
    """Shapes of the warp-per-system path (M >= N, M <= 32, N + nrhs <= 32) with padding, singular
    members and a batch that is not a multiple of the warps per CTA."""
    t, m, n, nrhs = shape
    lda, ldc, batch = m + 2, max(m, n) + 3, 23
    rng = np.random.default_rng(m * 131 + n * 7 + nrhs)
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    c = rng.standard_normal((batch, nrhs, ldc)).astype(np.float32)
    a[4] = 0.0
    a[5, 0, :] = 0.0
    check(handle, t, a, c, m, n, nrhs, lda, ldc, f"{t} {m}x{n}x{nrhs}")


def test_gels_large_batch(handle):
    row = ("big", "N", 32, 16, 2, 32, 32, 4096, "RANDOM", "-", "SUCCESS", "overdetermined")
    a, c = gels_inputs(row, 5)
    check(handle, "N", a, c, 32, 16, 2, 32, 32, "batch 4096")
