"""GPU checks of the strided-batch extensions and the pointer-array builder: the strided calls
give bit for bit what the pointer-array calls give on the same matrices."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


def test_build_pointer_array(ob, handle):
    import torch

    base = torch.zeros(1000, device="cuda")
    out = torch.zeros(37, dtype=torch.int64, device="cuda")
    assert ob.lib().aclblasBuildPointerArray(handle.h, C.c_void_p(base.data_ptr()), 100, 37,
                                             C.c_void_p(out.data_ptr())) == ob.SUCCESS
    torch.cuda.synchronize()
    want = base.data_ptr() + 100 * np.arange(37, dtype=np.int64)
    assert np.array_equal(out.cpu().numpy(), want)


@pytest.mark.parametrize("n", [8, 32, 48, 100])
def test_strided_chain_equals_pointer_array_chain(ob, handle, n):
    import torch

    L = ob.lib()
    batch, nrhs, lda = 300, 3, n + 2
    rng = np.random.default_rng(n)
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    b = rng.standard_normal((batch, nrhs, lda)).astype(np.float32)
    A1, B1 = to_dev(a, "cuda"), to_dev(b, "cuda")
    A2, B2 = A1.clone(), B1.clone()
    piv1, info1 = handle.getrf(A1, n, lda)
    handle.getrs("N", A1, n, lda, piv1, B1, nrhs, lda)
    C1 = torch.zeros((batch, n, n), device="cuda")
    rinfo1 = handle.getri(A1, n, lda, piv1, C1, n)

    piv2 = torch.zeros((batch, n), dtype=torch.int32, device="cuda")
    info2 = torch.zeros(batch, dtype=torch.int32, device="cuda")
    st = L.aclblasSgetrfStridedBatched(handle.h, n, C.c_void_p(A2.data_ptr()), lda, n * lda,
                                       C.c_void_p(piv2.data_ptr()), C.c_void_p(info2.data_ptr()), batch)
    assert st == ob.SUCCESS
    hinfo = C.c_int(-5)
    st = L.aclblasSgetrsStridedBatched(handle.h, ob.OP_N, n, nrhs, C.c_void_p(A2.data_ptr()), lda, n * lda,
                                       C.c_void_p(piv2.data_ptr()), C.c_void_p(B2.data_ptr()), lda, nrhs * lda,
                                       C.byref(hinfo), batch)
    assert st == ob.SUCCESS and hinfo.value == 0
    C2 = torch.zeros((batch, n, n), device="cuda")
    rinfo2 = torch.zeros(batch, dtype=torch.int32, device="cuda")
    st = L.aclblasSgetriStridedBatched(handle.h, n, C.c_void_p(A2.data_ptr()), lda, n * lda,
                                       C.c_void_p(piv2.data_ptr()), C.c_void_p(C2.data_ptr()), n, n * n,
                                       C.c_void_p(rinfo2.data_ptr()), batch)
    assert st == ob.SUCCESS
    torch.cuda.synchronize()
    for x, y in ((A1, A2), (B1, B2), (C1, C2)):
        assert torch.equal(x.view(torch.int32), y.view(torch.int32))
    assert torch.equal(piv1, piv2) and torch.equal(info1, info2) and torch.equal(rinfo1, rinfo2)
