"""GPU parity of aclblasSmatinvBatched (one fused launch) through the C ABI.

Expected values: the oracle's getrf on a copy of A followed by its getri (pinned to the
reference's matinv golden in test_matinv_oracle.py), bit for bit -- Ainv including what stays
outside the n x n block, and info. At the bench's scale the fused call is compared with the
library's own aclblasSgetrfBatched + aclblasSgetriBatched, also bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from cases import MATINV_CASES, MATINV_SEED
from conftest import to_dev, to_host
from test_lu_gpu import assert_bitwise
from test_matinv_oracle import oracle_matinv

pytestmark = pytest.mark.gpu


def gpu_matinv(handle, a, n, lda, lda_inv):
    import torch

    A = to_dev(a, "cuda")
    Ainv = torch.full((a.shape[0], max(1, n), lda_inv), -7.0, dtype=torch.float32, device="cuda")
    info = handle.matinv(A, n, lda, Ainv, lda_inv)
    torch.cuda.synchronize()
    assert np.array_equal(to_host(A), a), "A must not be modified"
    return to_host(Ainv), to_host(info)


@pytest.mark.parametrize("c", MATINV_CASES, ids=lambda c: c[0])
def test_matinv_csv(handle, c):
    name, n, lda, lda_inv, batch, mtype = c
    a = O.case_matrices(n, lda, mtype, MATINV_SEED, batch)
    cm, info = gpu_matinv(handle, a, n, lda, lda_inv)
    oc, oinfo = oracle_matinv(a, n, lda, lda_inv)
    np.testing.assert_array_equal(info, oinfo)
    assert_bitwise(cm, oc, name)


@pytest.mark.parametrize("n", range(1, 33))
def test_matinv_every_n_with_singular_members(handle, n):
    """Every size, a batch that is not a multiple of the per-CTA count, padded leading
    dimensions, and singular members: a zero column, two zero diagonal candidates, a zero
    matrix."""
    rng = np.random.default_rng(100 + n)
    batch, lda, lda_inv = 37, n + 3, n + 5
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    a[:, :, n:] = 9.0
    a[3, n // 2, :n] = 0.0          # column n/2 of matrix 3
    a[5] = 0.0                      # all zero
    if n > 2:
        a[7, :, :n] = np.triu(a[7, :, :n])  # triangular, with two zero diagonal entries
        a[7, 1, 1] = 0.0
        a[7, n - 1, n - 1] = 0.0
    cm, info = gpu_matinv(handle, a, n, lda, lda_inv)
    oc, oinfo = oracle_matinv(a, n, lda, lda_inv)
    np.testing.assert_array_equal(info, oinfo)
    assert info[5] > 0
    assert_bitwise(cm, oc, f"n={n}")


def test_matinv_in_place(handle):
    """A and Ainv the same matrices (lda == lda_inv): the same result as out of place."""
    import torch

    n, batch = 24, 300
    rng = np.random.default_rng(7)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    A = to_dev(a, "cuda")
    info = handle.matinv(A, n, n, A, n)
    torch.cuda.synchronize()
    oc, oinfo = oracle_matinv(a, n, n, n)
    np.testing.assert_array_equal(to_host(info), oinfo)
    assert_bitwise(to_host(A), oc, "in place")


def test_matinv_equals_getrf_getri_at_bench_scale(handle):
    """n = 32, 131072 matrices (512 MiB): the fused call equals the two-call sequence bit for
    bit; A * Ainv ~ I on a sample."""
    import torch

    n, batch = 32, 131072
    g = torch.Generator(device="cuda").manual_seed(11)
    A = torch.randn((batch, n, n), device="cuda", generator=g)
    Ainv = torch.empty_like(A)
    info = handle.matinv(A, n, n, Ainv, n)
    LU = A.clone()
    piv, finfo = handle.getrf(LU, n, n)
    C = torch.empty_like(A)
    rinfo = handle.getri(LU, n, n, piv, C, n)
    torch.cuda.synchronize()
    assert int(finfo.max()) == 0
    assert torch.equal(info, rinfo)
    assert torch.equal(Ainv.view(torch.int32), C.view(torch.int32))
    idx = torch.arange(0, batch, 4099, device="cuda")
    # column-major storage: the tensors hold A^T and Ainv^T, and Ainv^T A^T = (A Ainv)^T
    prod = torch.bmm(Ainv[idx].double(), A[idx].double())
    eye = torch.eye(n, dtype=torch.float64, device="cuda").expand_as(prod)
    res = torch.linalg.matrix_norm(prod - eye) / (
        torch.linalg.matrix_norm(A[idx].double()) * torch.linalg.matrix_norm(Ainv[idx].double()))
    assert float(res.max()) < 1e-5
