"""GPU parity of aclblasSgeqrfBatched through the C ABI: bit for bit against the oracle's
restatement (pinned to the reference's LAPACK golden in test_geqrf_oracle.py), on every success
row of the reference's geqrf CSV, on a sweep of shapes through both kernels (m, n <= 32: a warp
per matrix; otherwise a CTA per matrix), with padded leading dimensions left untouched, and at
the chain's scale (n = 32, 131072 matrices) through the reconstruction Q R = A."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import GEQRF_ROWS, geqrf_matrices
from conftest import to_dev, to_host
from test_geqrf_oracle import qr_reconstruct
from test_lu_gpu import assert_bitwise

pytestmark = pytest.mark.gpu


def gpu_geqrf(handle, a, m, n, lda):
    import torch

    A = to_dev(a, "cuda")
    tau = handle.geqrf(A, m, n, lda)
    torch.cuda.synchronize()
    return to_host(A), to_host(tau)


def check(handle, a, m, n, lda, what):
    x, t = gpu_geqrf(handle, a, m, n, lda)
    ox = a.copy()
    ot = O.port_geqrf(ox, m, n, lda)
    assert_bitwise(x, ox, what + " A")
    assert_bitwise(t[:, :min(m, n)], ot[:, :min(m, n)], what + " tau")


@pytest.mark.parametrize("row", [r for r in GEQRF_ROWS if r[8] == "SUCCESS" and min(r[1], r[2], r[4]) > 0],
                         ids=lambda r: r[0])
def test_geqrf_csv(handle, row):
    name, m, n, lda, batch, fill = row[:6]
    check(handle, geqrf_matrices(m, n, lda, fill, 7, batch), m, n, lda, name)


@pytest.mark.parametrize("mn", [(1, 1), (2, 7), (7, 2), (5, 5), (13, 31), (31, 13), (32, 32), (32, 1), (1, 32),
                                (17, 32), (32, 17), (33, 33), (40, 8), (8, 40), (100, 30), (30, 100)])
def test_geqrf_shapes_with_padding(handle, mn):
    m, n = mn
    lda, batch = m + 3, 37
    a = geqrf_matrices(m, n, lda, "RANDOM_NORM_2", 100 + m * 64 + n, batch)
    a[5, :, :m] = 0.0  # zero matrix: every tau 0
    if n > 1:
        a[6, 1, :m] = 0.0  # a zero column
    check(handle, a, m, n, lda, f"{m}x{n}")


def test_geqrf_chain_scale_reconstruction(handle):
    import torch

    m = n = 32
    batch = 131072
    g = torch.Generator(device="cuda").manual_seed(3)
    A0 = torch.randn((batch, n, m), device="cuda", generator=g)
    A = A0.clone()
    tau = handle.geqrf(A, m, n, m)
    torch.cuda.synchronize()
    x, t, a0 = to_host(A), to_host(tau), to_host(A0)
    for b in range(0, batch, 8191):
        ref = a0[b].T.astype(np.float64)
        err = np.linalg.norm(qr_reconstruct(x[b], t[b], m, n) - ref) / np.linalg.norm(ref)
        assert err < 1e-5, (b, err)
    sample = slice(0, 64)
    ox = a0[sample].copy()
    ot = O.port_geqrf(ox, m, n, m)
    assert_bitwise(x[sample], ox, "A sample")
    assert_bitwise(t[sample], ot, "tau sample")
