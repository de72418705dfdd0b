"""GPU parity of the batched LU chain through the C ABI (libopsblas_b200.so).

Two references:
  * the CPU oracle (oracle/lu_oracle.c, the reference kernels restated with one fmaf per
    update and true division): the CUDA kernels follow the same operation order, so factors,
    pivots, info, solutions and inverses must agree BIT FOR BIT;
  * the reference's own golden outputs (tests/golden/*.npz, LAPACK through the reference's
    golden headers): info exact, pivots exact when untied, factors under the reference's
    MIXED_TOLERANCE rule and 1e-5 normwise, solutions within the conditioning bound.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle as O
from cases import GETRF, GETRI, GETRS
from conftest import to_dev, to_host
from test_oracle_pin import GOLD, NORMWISE, TIE, c1_inputs, solution_ok

pytestmark = pytest.mark.gpu


def gpu_getrf(handle, a, n, lda, pivot=True):
    import torch

    A = to_dev(a, "cuda")
    piv, info = handle.getrf(A, n, lda, pivot=pivot)
    torch.cuda.synchronize()
    return to_host(A), (to_host(piv) if pivot else None), to_host(info)


def gpu_getrs(handle, trans, lu, n, lda, piv, b, nrhs, ldb):
    import torch

    LU = to_dev(lu, "cuda")
    B = to_dev(b, "cuda")
    P = to_dev(piv, "cuda") if piv is not None else None
    info = handle.getrs(trans, LU, n, lda, P, B, nrhs, ldb)
    torch.cuda.synchronize()
    return to_host(B), info


def gpu_getri(handle, lu, n, lda, piv, ldc):
    import torch

    LU = to_dev(lu, "cuda")
    P = to_dev(piv, "cuda") if piv is not None else None
    Cm = torch.full((lu.shape[0], max(1, n), ldc), -7.0, dtype=torch.float32, device="cuda")
    info = handle.getri(LU, n, lda, P, Cm, ldc)
    torch.cuda.synchronize()
    return to_host(Cm), to_host(info)


def assert_bitwise(x, y, what):
    """Bit-for-bit equality; NaNs compare equal whatever their payload (CPU and GPU NaNs
    carry different payloads)."""
    xa, ya = np.ascontiguousarray(x), np.ascontiguousarray(y)
    xb, yb = xa.view(np.uint32).ravel(), ya.view(np.uint32).ravel()
    both_nan = np.isnan(xa).ravel() & np.isnan(ya).ravel()
    bad = np.flatnonzero((xb != yb) & ~both_nan)
    assert bad.size == 0, f"{what}: {bad.size} elements differ, first at {bad[:5]}: " \
                          f"{x.ravel()[bad[:5]]} vs {y.ravel()[bad[:5]]}"


# ------------------------------------------------------------------------- parity config --

def test_c1_getrf_getrs_vs_golden_and_oracle(handle):
    """n = 16, 1024 matrices, N(0,1), nrhs = 1 (the parity configuration)."""
    g = np.load(os.path.join(GOLD, "c1.npz"))
    A, B = c1_inputs()
    lu, piv, info = gpu_getrf(handle, A, 16, 16)
    olu = A.copy()
    opiv, oinfo, gap = O.port_getrf(olu, 16, 16)
    assert_bitwise(lu, olu, "LU vs oracle")
    np.testing.assert_array_equal(piv, opiv)
    np.testing.assert_array_equal(info, oinfo)
    # against the reference golden
    np.testing.assert_array_equal(info, g["info"])
    untied = gap >= TIE
    np.testing.assert_array_equal(piv[untied], g["piv"][untied])
    for b in range(len(g["LU"])):
        assert O.mixed_tolerance_ok(lu[b], g["LU"][b]) and O.normwise_rel(lu[b], g["LU"][b]) <= NORMWISE
    x, hinfo = gpu_getrs(handle, "N", lu, 16, 16, piv, B, 1, 16)
    assert hinfo == 0
    ox = B.copy()
    O.port_getrs("N", olu, 16, 16, opiv, ox, 1, 16)
    assert_bitwise(x, ox, "X vs oracle")
    for b in range(1024):
        assert solution_ok(x[b].T, g["X"][b].T, A[b], B[b].T), b


# ------------------------------------------------------------------ reference CSV suites --

@pytest.mark.parametrize("c", [c for c in GETRF if c.status == "SUCCESS"], ids=lambda c: c.name)
def test_getrf_csv(handle, c):
    if c.n == 0 or c.batch == 0:
        return  # no-op rows: covered by test_noop_calls_touch_nothing
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    lu, piv, info = gpu_getrf(handle, a, c.n, c.lda, c.pivot)
    olu = a.copy()
    opiv, oinfo, _ = O.port_getrf(olu, c.n, c.lda, c.pivot)
    assert_bitwise(lu, olu, "LU")
    np.testing.assert_array_equal(info, oinfo)
    if c.pivot:
        np.testing.assert_array_equal(piv, opiv)


@pytest.mark.parametrize("c", [c for c in GETRS if c.status == "SUCCESS" and c.n > 0 and c.nrhs > 0
                               and c.batch > 0], ids=lambda c: c.name)
def test_getrs_csv(handle, c):
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    b = O.case_rhs(c.n, c.nrhs, c.ldb, c.seed, c.batch)
    piv, _, _ = O.port_getrf(a, c.n, c.lda, c.pivot)
    x, hinfo = gpu_getrs(handle, c.trans, a, c.n, c.lda, piv if c.pivot else None, b, c.nrhs, c.ldb)
    assert hinfo == 0
    ox = b.copy()
    O.port_getrs(c.trans, a, c.n, c.lda, piv if c.pivot else None, ox, c.nrhs, c.ldb)
    assert_bitwise(x, ox, "X")


@pytest.mark.parametrize("n", list(range(1, 33)))
def test_getrs_transposed_single_rhs_bitwise(handle, n):
    """trans T / C with one right-hand side at every n <= 32 (padded lda and ldb, a batch that
    is not a multiple of the per-CTA count): the U^T and L^T sweeps add each x[j]'s terms in the
    reference's order, so X equals the oracle bit for bit."""
    rng = np.random.default_rng(300 + n)
    batch, lda, ldb = 37, n + 1, n + 2
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    piv, _, _ = O.port_getrf(a, n, lda)
    b = rng.standard_normal((batch, 1, ldb)).astype(np.float32)
    for trans in ("T", "C"):
        x, hinfo = gpu_getrs(handle, trans, a, n, lda, piv, b, 1, ldb)
        assert hinfo == 0
        ox = b.copy()
        O.port_getrs(trans, a, n, lda, piv, ox, 1, ldb)
        assert_bitwise(x, ox, f"X {trans} n={n}")


@pytest.mark.parametrize("c", [c for c in GETRI if c.status == "SUCCESS" and c.n > 0 and c.batch > 0],
                         ids=lambda c: c.name)
def test_getri_csv(handle, c):
    a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
    piv, _, _ = O.port_getrf(a, c.n, c.lda, c.pivot)
    cm, info = gpu_getri(handle, a, c.n, c.lda, piv if c.pivot else None, c.ldc)
    oc = np.full((c.batch, c.n, c.ldc), -7.0, np.float32)
    oinfo = O.port_getri(a, c.n, c.lda, piv if c.pivot else None, oc, c.ldc)
    np.testing.assert_array_equal(info, oinfo)
    assert_bitwise(cm, oc, "C")


# -------------------------------------------------------------------------- edge cases --

@pytest.mark.parametrize("n", list(range(1, 33)) + [33, 40, 64, 100, 128, 129, 160, 300])
def test_getrf_every_small_n_with_tail_and_padding(handle, n):
    """Every register-kernel size, a batch that is not a multiple of the per-CTA matrix count,
    lda > n with sentinel padding that must survive untouched."""
    rng = np.random.default_rng(n)
    batch, lda = 37, n + 3
    a = rng.standard_normal((batch, n, lda)).astype(np.float32)
    a[:, :, n:] = 12345.0
    lu, piv, info = gpu_getrf(handle, a, n, lda)
    olu = a.copy()
    opiv, oinfo, _ = O.port_getrf(olu, n, lda)
    assert_bitwise(lu, olu, "LU")
    np.testing.assert_array_equal(piv, opiv)
    np.testing.assert_array_equal(info, oinfo)
    assert np.all(lu[:, :, n:] == 12345.0)


@pytest.mark.parametrize("n", [1, 3, 8, 16, 31, 32, 48, 150])
def test_singular_nan_and_zero_pivots(handle, n):
    """Zero columns (info, zeroed trailing pivots), a NaN entry (never chosen as pivot), and
    exact ties (lowest row wins), bit-exact against the oracle."""
    rng = np.random.default_rng(100 + n)
    batch = 8
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    a[1, min(2, n - 1), :] = 0.0                      # zero column -> info
    a[2, 0, :] = 0.0
    a[3, 0, min(1, n - 1)] = np.nan                   # NaN candidate
    a[4, 0, :] = 1.0                                  # all-equal first column: tie -> row 0
    a[5] = np.round(a[5])                             # many exact ties
    lu, piv, info = gpu_getrf(handle, a, n, n)
    olu = a.copy()
    opiv, oinfo, _ = O.port_getrf(olu, n, n)
    assert_bitwise(lu, olu, "LU")
    np.testing.assert_array_equal(piv, opiv)
    np.testing.assert_array_equal(info, oinfo)
    assert info[2] == 1 and np.all(piv[2, 1:] == 0)


@pytest.mark.parametrize("n", [5, 16, 32, 64])
def test_no_pivot_without_info(handle, n, ob):
    """PivotArray == NULL and infoArray == NULL is legal (no-pivot mode)."""
    import torch

    rng = np.random.default_rng(7)
    a = (rng.standard_normal((9, n, n)) + 4 * n * np.eye(n)).astype(np.float32)
    A = to_dev(a, "cuda")
    aptr = ob.ptr_array(A)  # kept referenced until the launch is enqueued
    st = ob.lib().aclblasSgetrfBatched(handle.h, n, aptr.data_ptr(), n, None, None, 9)
    assert st == ob.SUCCESS
    torch.cuda.synchronize()
    olu = a.copy()
    O.port_getrf(olu, n, n, pivot=False)
    assert_bitwise(to_host(A), olu, "LU")


def test_noop_calls_touch_nothing(handle, ob):
    L = ob.lib()
    assert L.aclblasSgetrfBatched(handle.h, 0, None, 1, None, None, 4) == ob.SUCCESS
    assert L.aclblasSgetrfBatched(handle.h, 32, None, 32, None, None, 0) == ob.SUCCESS
    assert L.aclblasSgetriBatched(handle.h, 0, None, 1, None, None, 1, None, 4) == ob.SUCCESS
    import ctypes as C

    info = C.c_int(-1)
    assert L.aclblasSgetrsBatched(handle.h, ob.OP_N, 32, 0, None, 32, None, None, 32, C.byref(info), 4) == 0
    assert info.value == 0


def test_getrs_nrhs_chunks_and_ldb(handle):
    """nrhs that is not a multiple of the 4-column chunk, ldb > n, both transposes."""
    rng = np.random.default_rng(3)
    for n, nrhs in [(7, 3), (16, 5), (32, 9), (32, 256), (33, 6), (12, 1), (31, 2), (30, 4)]:
        a = rng.standard_normal((11, n, n)).astype(np.float32)
        piv, _, _ = O.port_getrf(a, n, n)
        b = rng.standard_normal((11, nrhs, n + 2)).astype(np.float32)
        for trans in ("N", "T"):
            x, _ = gpu_getrs(handle, trans, a, n, n, piv, b, nrhs, n + 2)
            ox = b.copy()
            O.port_getrs(trans, a, n, n, piv, ox, nrhs, n + 2)
            if trans == "N" or n > 32 or nrhs > 1:
                assert_bitwise(x, ox, f"X n={n} nrhs={nrhs} {trans}")
            else:
                np.testing.assert_allclose(x, ox, rtol=2e-4, atol=1e-5)
            assert np.all(x[:, :, n:] == b[:, :, n:])


def test_getri_singular_semantics(handle):
    """Highest zero diagonal reported; C content on failure follows the reference per n."""
    rng = np.random.default_rng(5)
    for n in (4, 8, 9, 16, 40):
        lu = rng.standard_normal((4, n, n)).astype(np.float32)
        lu[1, n // 2, n // 2] = 0.0
        lu[2, 0, 0] = 0.0
        lu[2, n - 1, n - 1] = 0.0
        piv = np.tile(np.arange(1, n + 1, dtype=np.int32), (4, 1))
        piv[:, 0] = 2
        cm, info = gpu_getri(handle, lu, n, n, piv, n)
        oc = np.full((4, n, n), -7.0, np.float32)
        oinfo = O.port_getri(lu, n, n, piv, oc, n)
        np.testing.assert_array_equal(info, oinfo)
        assert info[2] == n
        assert_bitwise(cm, oc, f"C n={n}")


# --------------------------------------------------------- the chain at scale (n = 32) --

def test_chain_n32_at_scale_properties(handle):
    """n = 32, 131072 matrices, A ~ N(0,1), B ~ U(-1,1), nrhs = 4: getrf -> getrs -> getri.
    Size-independent checks on the whole batch (backward error of X, A * inv(A) = I, bitwise
    determinism across runs) and bit-exact oracle parity on a sample of matrices."""
    import torch

    n, batch, nrhs = 32, 131072, 4
    g = torch.Generator(device="cuda").manual_seed(1)
    A0 = torch.randn((batch, n, n), device="cuda", generator=g)
    B0 = torch.rand((batch, nrhs, n), device="cuda", generator=g) * 2 - 1
    LU = A0.clone()
    piv, info = handle.getrf(LU, n, n)
    X = B0.clone()
    handle.getrs("N", LU, n, n, piv, X, nrhs, n)
    Cinv = torch.empty_like(A0)
    rinfo = handle.getri(LU, n, n, piv, Cinv, n)
    LU2 = A0.clone()
    piv2, _ = handle.getrf(LU2, n, n)
    torch.cuda.synchronize()
    assert torch.equal(LU, LU2) and torch.equal(piv, piv2)
    assert int(info.max()) == 0 and int(rinfo.max()) == 0
    # backward error of X in FP64, column-major: math A = A0[b].T
    Am = A0.double().transpose(1, 2)
    R = B0.double().transpose(1, 2) - Am @ X.double().transpose(1, 2)
    den = Am.abs().sum(2).amax(1) * X.double().abs().amax((1, 2)) + B0.double().abs().amax((1, 2))
    berr = R.abs().amax((1, 2)) / den
    assert float(berr.max()) < 1e-5
    # a column-wise backward-stable inverse satisfies ||A C - I|| <= c n eps ||A|| ||C||
    Cm = Cinv.double().transpose(1, 2)
    E = Am @ Cm - torch.eye(n, device="cuda", dtype=torch.float64)
    scale = Am.abs().sum(2).amax(1) * Cm.abs().sum(2).amax(1)
    assert float((E.abs().sum(2).amax(1) / scale).max()) < 1e-5
    # bit-exact parity on a sample
    idx = torch.randperm(batch, generator=torch.Generator().manual_seed(0))[:256].numpy()
    a = to_host(A0)[idx].copy()
    opiv, oinfo, _ = O.port_getrf(a, n, n)
    assert_bitwise(to_host(LU)[idx], a, "LU sample")
    np.testing.assert_array_equal(to_host(piv)[idx], opiv)
    ox = to_host(B0)[idx].copy()
    O.port_getrs("N", a, n, n, opiv, ox, nrhs, n)
    assert_bitwise(to_host(X)[idx], ox, "X sample")
    oc = np.zeros_like(a)
    O.port_getri(a, n, n, opiv, oc, n)
    assert_bitwise(to_host(Cinv)[idx], oc, "C sample")


def test_error_rows_with_real_handle(handle, ob):
    """The validation paths behave the same with a live handle."""
    import ctypes as C

    import torch

    L = ob.lib()
    # small real device buffers: the calls are rejected before they are read, and stay untouched
    bufs = [torch.zeros(64, dtype=torch.float64, device="cuda") for _ in range(2)]
    P = [C.c_void_p(t.data_ptr()) for t in bufs]
    assert L.aclblasSgetrfBatched(handle.h, 5, P[0], 3, None, None, 4) == ob.INVALID_VALUE
    info = C.c_int(0)
    assert L.aclblasSgetrsBatched(handle.h, 999, 4, 1, None, 4, None, None, 4, C.byref(info), 1) == ob.INVALID_ENUM
    assert info.value == -2
    assert L.aclblasSgetriBatched(handle.h, 4, P[0], 4, None, P[1], 4, None, 1) == ob.INVALID_VALUE
    torch.cuda.synchronize()
    assert all(float(t.abs().sum()) == 0.0 for t in bufs)


def test_handle_stream_and_workspace(ob, cuda):
    import ctypes as C

    import torch

    L = ob.lib()
    h = C.c_void_p()
    assert L.aclblasCreate(C.byref(h)) == ob.SUCCESS
    s = torch.cuda.Stream()
    assert L.aclblasSetStream(h, C.c_void_p(s.cuda_stream)) == ob.SUCCESS
    got = C.c_void_p()
    assert L.aclblasGetStream(h, C.byref(got)) == ob.SUCCESS and got.value == s.cuda_stream
    ws = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    assert L.aclblasSetWorkspace(h, C.c_void_p(ws.data_ptr()), ws.numel()) == ob.SUCCESS
    assert L.aclblasSetWorkspace(h, C.c_void_p(ws.data_ptr()), 16) == ob.SUCCESS  # grow-only: ignored
    assert L.aclblasSetStream(h, None) == ob.SUCCESS  # back to the library workspace
    assert L.aclblasDestroy(h) == ob.SUCCESS


def test_unaligned_matrices_take_the_scalar_paths(handle, ob):
    """Matrices whose addresses are 4- but not 16-byte aligned (and lda not a multiple of 4)
    use the element-wise staging paths; results must not change."""
    import torch

    rng = np.random.default_rng(11)
    for n, lda, nrhs in [(32, 32, 4), (16, 17, 3), (8, 8, 2)]:
        batch = 19
        a = rng.standard_normal((batch, n, lda)).astype(np.float32)
        piv, _, _ = O.port_getrf(a, n, lda)
        b = rng.standard_normal((batch, nrhs, n)).astype(np.float32)
        # one extra float in front of every matrix: element stride lda*n + 1
        flat = np.zeros((batch, n * lda + 1), np.float32)
        flat[:, 1:] = a.reshape(batch, -1)
        fb = np.zeros((batch, nrhs * n + 1), np.float32)
        fb[:, 1:] = b.reshape(batch, -1)
        A = to_dev(flat, "cuda")
        Bd = to_dev(fb, "cuda")
        P = to_dev(piv, "cuda")
        aptr = ob.ptr_array(A) + 4
        bptr = ob.ptr_array(Bd) + 4
        for trans in ("N", "T"):
            Bd.copy_(to_dev(fb, "cuda"))
            handle.getrs(trans, A, n, lda, P, Bd, nrhs, n, aptr=aptr, bptr=bptr)
            torch.cuda.synchronize()
            x = to_host(Bd)[:, 1:].reshape(batch, nrhs, n)
            ox = b.copy()
            O.port_getrs(trans, a, n, lda, piv, ox, nrhs, n)
            assert_bitwise(x, ox, f"getrs {trans} n={n}")
        Cm = torch.zeros((batch, n * n + 1), dtype=torch.float32, device="cuda")
        cptr = ob.ptr_array(Cm) + 4
        info = handle.getri(A, n, lda, P, Cm, n, aptr=aptr, cptr=cptr)
        torch.cuda.synchronize()
        oc = np.zeros((batch, n, n), np.float32)
        oinfo = O.port_getri(a, n, lda, piv, oc, n)
        assert_bitwise(to_host(Cm)[:, 1:].reshape(batch, n, n), oc, f"getri n={n}")
        np.testing.assert_array_equal(to_host(info), oinfo)


@pytest.mark.parametrize("n,batch", [(48, 8192), (128, 4096), (160, 2048), (256, 2048)])
def test_getrf_getrs_full_occupancy(handle, n, batch):
    """Batches that fill every SM several times over (where CTAs of one kernel share SMs and
    any missing barrier shows): a random sample is bit-identical to the oracle, and every
    matrix's solution has an FP64 backward error at FP32 level."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(n)
    A0 = torch.randn(batch, n, n, device="cuda", generator=g)
    B0 = torch.randn(batch, 2, n, device="cuda", generator=g)
    LU, X = A0.clone(), B0.clone()
    piv, info = handle.getrf(LU, n, n)
    handle.getrs("N", LU, n, n, piv, X, 2, n)
    torch.cuda.synchronize()
    assert int(info.max()) == 0
    a64 = A0.double().transpose(1, 2)
    x64 = X.double().transpose(1, 2)
    b64 = B0.double().transpose(1, 2)
    r = b64 - a64 @ x64
    an = a64.abs().sum(2).amax(1)
    berr = (r.abs().amax(1) / (an[:, None] * x64.abs().amax(1) + b64.abs().amax(1))).amax(1)
    assert float(berr.max()) < 1e-5, float(berr.max())
    sample = np.random.default_rng(n).choice(batch, 24, replace=False)
    a = to_host(A0)[sample].copy()
    opiv, oinfo, _ = O.port_getrf(a, n, n)
    np.testing.assert_array_equal(to_host(piv)[sample], opiv)
    assert np.array_equal(to_host(LU)[sample].view(np.uint32), a.view(np.uint32))
