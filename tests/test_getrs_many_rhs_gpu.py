"""aclblasSgetrsBatched, trans N, 32 < n <= 128 with at least 65536 right-hand sides in the batch:
one thread per right-hand side walking LU columns. Bit for bit against the oracle, for a packed
16-byte-aligned layout and a padded odd leading dimension (the per-element load path), with some
matrices skipped through a NULL right-hand-side pointer."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import to_dev, to_host
from test_lu_gpu import assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,nrhs,batch,pad", [(64, 8, 8192, 0), (33, 1, 65536, 0), (100, 2, 32768, 3),
                                              (128, 4, 16384, 0)])
def test_getrs_many_rhs_trans_n(handle, n, nrhs, batch, pad):
    import torch

    lda = ldb = n + pad
    rng = np.random.default_rng(n * 7 + nrhs)
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    lu = a.copy()
    piv, _, _ = O.port_getrf(lu, n, lda)
    b = rng.standard_normal((batch, nrhs, ldb)).astype(np.float32)
    want = b.copy()
    O.port_getrs("N", lu, n, lda, piv, want, nrhs, ldb)
    LU, B = to_dev(lu, "cuda"), to_dev(b, "cuda")
    bptr = torch.arange(batch, device="cuda", dtype=torch.int64) * (nrhs * ldb * 4) + B.data_ptr()
    skip = torch.arange(0, batch, 97, device="cuda")
    bptr[skip] = 0  # NULL right-hand side: the matrix is skipped
    handle.getrs("N", LU, n, lda, to_dev(piv, "cuda"), B, nrhs, ldb, bptr=bptr)
    torch.cuda.synchronize()
    got = to_host(B)
    keep = np.ones(batch, bool)
    keep[np.arange(0, batch, 97)] = False
    assert_bitwise(got[keep], want[keep], f"n={n} nrhs={nrhs}")
    assert np.array_equal(got[~keep], b[~keep])
