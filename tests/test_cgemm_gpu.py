"""GPU parity of aclblasCgemmBatched through the C ABI.

Expected values: the oracle's restatement (pinned to the reference's Cgemm golden in
test_cgemm_oracle.py), bit for bit -- the device kernel forms the same four FP32 sums (one fmaf
per product, k in order) and the reference's combine with the same roundings. Every success row
of the reference's Cgemm CSV; C beyond row m untouched; a null C pointer skips its matrix;
alpha == 0 reads neither A nor B; at the bench's shape a sample of matrices is checked.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import to_dev, to_host
from test_cgemm_oracle import PAD, VALUE_ROWS, cgemm_inputs

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x).view(np.uint32)


def gpu_cgemm(handle, c, a, b, cm, cptr=None):
    import torch

    name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = c
    Cd = to_dev(cm, "cuda")
    handle.cgemm(ta, tb, m, n, k, alpha, to_dev(a, "cuda"), lda, to_dev(b, "cuda"), ldb, beta, Cd, ldc, cptr=cptr)
    torch.cuda.synchronize()
    return to_host(Cd)


@pytest.mark.parametrize("c", VALUE_ROWS, ids=lambda c: c[0])
def test_cgemm_csv_bitexact(handle, c):
    name, ta, tb, m, n, k, alpha, beta, lda, ldb, ldc, batch, cfill = c
    a, b, cm = cgemm_inputs(c)
    got = gpu_cgemm(handle, c, a, b, cm)
    want = cm.copy()
    O.port_cgemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, want, ldc)
    assert np.all(got[:, :, m:] == PAD), "rows beyond m must be untouched"
    assert np.array_equal(_bits(got), _bits(want)), name


def test_cgemm_null_c_entry_skips_matrix(ob, handle):
    import torch

    c = ("nullc", "C", "T", 37, 29, 41, 0.5 - 1.5j, 0.25 + 0.5j, 41, 29, 40, 5, "R")
    a, b, cm = cgemm_inputs(c)
    Cd = to_dev(cm, "cuda")
    cptr = ob.ptr_array(Cd)
    cptr[2] = 0
    handle.cgemm("C", "T", 37, 29, 41, 0.5 - 1.5j, to_dev(a, "cuda"), 41, to_dev(b, "cuda"), 29, 0.25 + 0.5j, Cd, 40,
                 cptr=cptr)
    torch.cuda.synchronize()
    got = to_host(Cd)
    want = cm.copy()
    O.port_cgemm("C", "T", 37, 29, 41, 0.5 - 1.5j, a, 41, b, 29, 0.25 + 0.5j, want, 40, skip_c=(2,))
    assert np.array_equal(got[2], cm[2])
    assert np.array_equal(_bits(got), _bits(want))


def test_cgemm_alpha_zero_reads_no_operand(handle):
    """alpha == 0 with NaN operands: C = beta C exactly as the oracle's zero-sum combine."""
    c = ("azero", "N", "N", 70, 66, 19, 0j, 0.5 - 0.25j, 70, 19, 72, 3, "R")
    a, b, cm = cgemm_inputs(c)
    a[:] = np.nan
    b[:] = np.nan
    got = gpu_cgemm(handle, c, a, b, cm)
    want = cm.copy()
    O.port_cgemm("N", "N", 70, 66, 19, 0j, a, 70, b, 19, 0.5 - 0.25j, want, 72)
    assert np.all(np.isfinite(got[:, :, :70]))
    assert np.array_equal(_bits(got), _bits(want))


def test_cgemm_beta_zero_overwrites_nan(handle):
    c = ("bzero", "T", "C", 33, 65, 17, 1.25 + 0.5j, 0j, 17, 65, 33, 2, "R")
    a, b, cm = cgemm_inputs(c)
    cm[:, :, :33] = np.nan
    got = gpu_cgemm(handle, c, a, b, cm)
    want = cm.copy()
    O.port_cgemm("T", "C", 33, 65, 17, 1.25 + 0.5j, a, 17, b, 65, 0j, want, 33)
    assert np.all(np.isfinite(got))
    assert np.array_equal(_bits(got), _bits(want))


def test_cgemm_bench_shape_sample(handle):
    """64 x 64 x 64, 16384 matrices generated on the device: a sample of matrices bit for bit
    against the oracle."""
    import torch

    m = n = k = 64
    batch = 16384
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn((batch, k, m), dtype=torch.complex64, device="cuda", generator=g)
    B = torch.randn((batch, n, k), dtype=torch.complex64, device="cuda", generator=g)
    Cd = torch.randn((batch, n, m), dtype=torch.complex64, device="cuda", generator=g)
    C0 = Cd.clone()
    alpha, beta = 1.5 + 0.3j, 0.3 - 0.1j
    handle.cgemm("N", "N", m, n, k, alpha, A, m, B, k, beta, Cd, m)
    torch.cuda.synchronize()
    idx = [0, 1, 4097, 9999, batch - 1]
    a = A[idx].cpu().numpy()
    b = B[idx].cpu().numpy()
    want = C0[idx].cpu().numpy()
    O.port_cgemm("N", "N", m, n, k, alpha, a, m, b, k, beta, want, m)
    got = Cd[idx].cpu().numpy()
    assert np.array_equal(_bits(got), _bits(want))
