"""GPU tests of the device status word (aclblasGetDeviceStatus) that the kernels' bounded waits
report to.

A wait is made to give up through the library's test hook (opsblas_test_set_wait_limit: every
bounded wait launched afterwards polls at most the given number of times; 0 gives up at once).
Nothing faults or hangs: a kernel whose wait gave up stops issuing work, waits (with the normal
bound) for what it already has in flight, releases its tensor memory and returns. The call still
returns SUCCESS (it is asynchronous); the next aclblasGetDeviceStatus returns EXECUTION_FAILED
with the kernel's bit, the one after that is clean, and the handle keeps computing correct
results.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import to_dev, to_host

pytestmark = pytest.mark.gpu


def _hook(ob):
    f = ob.lib().opsblas_test_set_wait_limit
    f.argtypes = [C.c_uint]
    f.restype = None
    return f


def test_device_status_clean(ob, handle):
    st, flags = handle.device_status()
    assert st == ob.SUCCESS and flags == 0


def test_gemm_wait_gives_up_and_reports(ob, cuda):
    import torch

    hook = _hook(ob)
    m = n = k = 256
    batch = 4
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn((batch, k, m), device="cuda", generator=g).half()
    B = torch.randn((batch, n, k), device="cuda", generator=g).half()
    C0 = torch.randn((batch, n, m), device="cuda", generator=g).half()
    with ob.Handle() as h:
        Cm = C0.clone()
        hook(0)
        try:
            h.gemm_batched_ex("N", "N", m, n, k, 1.0, A, 1, m, B, 1, k, 0.0, Cm, 1, m, compute=ob.COMPUTE_32F)
            torch.cuda.synchronize()
        finally:
            hook(0xFFFFFFFF)
        st, flags = h.device_status()
        assert st == ob.EXECUTION_FAILED and flags & 4
        assert torch.equal(Cm, C0)  # C is left as it was
        st, flags = h.device_status()
        assert st == ob.SUCCESS and flags == 0
        h.gemm_batched_ex("N", "N", m, n, k, 1.0, A, 1, m, B, 1, k, 0.0, Cm, 1, m, compute=ob.COMPUTE_32F)
        torch.cuda.synchronize()
        ref = torch.bmm(B.float(), A.float())  # (A B)^T = B^T A^T in the (batch, cols, rows) storage
        err = (Cm.float() - ref).abs().max().item()
        assert err <= 4e-3 * ref.abs().max().item() + 1e-2
        st, flags = h.device_status()
        assert st == ob.SUCCESS and flags == 0


def test_tmem_lu_wait_gives_up_and_reports(ob, cuda):
    import torch

    hook = _hook(ob)
    n, nrhs, batch = 48, 2, 16
    rng = np.random.default_rng(4)
    a = (rng.standard_normal((batch, n, n)) + 8 * np.eye(n)).astype(np.float32)
    b = rng.standard_normal((batch, nrhs, n)).astype(np.float32)
    A, B = to_dev(a, "cuda"), to_dev(b, "cuda")
    with ob.Handle() as h:
        hook(0)
        try:
            _, _, _, info, _, _ = h.refine(A, B, n, nrhs, compute=ob.COMPUTE_32F_FAST_TF32, max_iter=2, tol=1e-6)
            torch.cuda.synchronize()
        finally:
            hook(0xFFFFFFFF)
        st, flags = h.device_status()
        assert st == ob.EXECUTION_FAILED and flags & 2
        assert (to_host(info) == -1).all()
        st, flags = h.device_status()
        assert st == ob.SUCCESS and flags == 0
        X, _, _, info, berr, _ = h.refine(A, B, n, nrhs, compute=ob.COMPUTE_32F_FAST_TF32, max_iter=5, tol=1e-6)
        torch.cuda.synchronize()
        assert int(to_host(info).max()) == 0 and float(to_host(berr).max()) <= 1e-6
        st, flags = h.device_status()
        assert st == ob.SUCCESS and flags == 0
