"""GPU tests of aclblasGemmBatchedEx, the refinement entry point and the solve adjoint."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import to_dev, to_host

pytestmark = pytest.mark.gpu


# ------------------------------------------------------------------------ GemmBatchedEx --

def _quantize(x, kind):
    import torch

    t = torch.from_numpy(x)
    if kind == "F16":
        return t.half()
    if kind == "BF16":
        return t.bfloat16()
    if kind == "E4M3":
        return t.to(torch.float8_e4m3fn)
    if kind == "E5M2":
        return t.to(torch.float8_e5m2)
    return t.float()


def _tf32(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x0FFF + ((u >> 13) & 1)) & 0xFFFFE000).astype(np.uint32)
    return u.view(np.float32)


GEMM_CASES = [
    # (ta, tb, m, n, k, alpha, beta, A, B, C, compute, rtol)
    ("N", "N", 128, 128, 128, 1.0, 0.0, "F16", "F16", "F16", 0, 4e-3),
    ("N", "T", 128, 128, 128, 1.0, 0.0, "F16", "F16", "F16", 2, 4e-3),
    ("T", "N", 64, 96, 80, 0.5, 0.5, "F16", "F16", "F16", 2, 4e-3),
    ("C", "C", 33, 17, 23, -1.0, -0.5, "F16", "F16", "F16", 0, 4e-3),
    ("N", "N", 17, 19, 23, 1.0, 0.0, "BF16", "BF16", "BF16", 2, 2e-2),
    ("N", "T", 128, 128, 128, 1.0, 1.0, "BF16", "BF16", "BF16", 2, 2e-2),
    ("N", "N", 128, 128, 128, 1.0, 0.0, "E4M3", "E4M3", "F16", 2, 4e-3),
    ("N", "N", 96, 64, 128, 1.0, 0.0, "E5M2", "E4M3", "F16", 2, 4e-3),
    ("N", "N", 64, 64, 64, 1.0, 0.0, "E4M3", "E5M2", "F16", 2, 4e-3),
    ("N", "N", 64, 64, 64, 1.0, 0.0, "E5M2", "E5M2", "F16", 2, 4e-3),
    ("N", "N", 100, 70, 50, 1.0, 0.0, "F32", "F32", "F32", 3, 1e-5),
    ("T", "N", 100, 70, 50, -1.0, 1.0, "F32", "F32", "F32", 6, 2e-3),
    ("N", "N", 300, 260, 100, 1.0, 0.5, "F32", "F32", "F32", 6, 2e-3),   # tcgen05: several tiles, ragged edges
    ("T", "T", 129, 257, 33, -2.0, 0.0, "F32", "F32", "F32", 6, 2e-3),
    ("N", "T", 128, 128, 8, 1.0, 1.0, "F32", "F32", "F32", 6, 2e-3),
    ("N", "T", 64, 64, 32, 1.0, 0.0, "F32", "F32", "F32", 5, 2e-2),
    # tcgen05 pipeline: several K tiles (more than the pipeline's stages), every orientation,
    # ragged edges, beta != 0 in the C type, and leading dimensions that are not 16-byte multiples
    # (register path instead of cp.async)
    ("N", "N", 200, 136, 520, 1.0, 0.0, "F16", "F16", "F16", 2, 4e-3),
    ("T", "T", 130, 250, 300, 0.75, -0.5, "F16", "F16", "F16", 2, 4e-3),
    ("T", "N", 256, 256, 256, 1.0, 1.0, "BF16", "BF16", "BF16", 2, 2e-2),
    ("N", "T", 77, 91, 333, -1.0, 0.25, "BF16", "BF16", "BF16", 2, 2e-2),
    ("T", "N", 160, 144, 512, 1.0, 0.0, "E4M3", "E4M3", "F16", 2, 4e-3),
    ("N", "T", 129, 130, 257, 1.0, 0.5, "E5M2", "E4M3", "F16", 2, 4e-3),
    ("T", "T", 96, 100, 200, 1.0, 0.0, "E4M3", "E5M2", "F16", 2, 4e-3),
    ("N", "N", 257, 129, 300, 1.0, 0.0, "F32", "F32", "F32", 6, 2e-3),
    ("T", "T", 140, 70, 130, 1.0, -1.0, "F32", "F32", "F32", 5, 2e-2),
    ("T", "N", 300, 260, 200, 1.0, 0.5, "F32", "F32", "F32", 6, 2e-3),   # FP32 by TMA, converted in shared memory
    ("T", "N", 128, 64, 36, -1.0, 1.0, "F32", "F32", "F32", 6, 2e-3),
]
DT = {"F32": 0, "F16": 1, "BF16": 27, "E5M2": 35, "E4M3": 36}


@pytest.mark.parametrize("case", GEMM_CASES, ids=lambda c: "_".join(map(str, c[:5] + c[7:11])))
def test_gemm_batched_ex_numerics(handle, case):
    import torch

    ta, tb, m, n, k, alpha, beta, at, bt, ct, comp, rtol = case
    batch = 3
    rng = np.random.default_rng(m * 7 + n)
    ra, ca = (k, m) if ta != "N" else (m, k)
    rb, cb = (n, k) if tb != "N" else (k, n)
    # column-major batches: tensor shape (batch, cols, rows)
    a = rng.uniform(-1, 1, (batch, ca, ra)).astype(np.float32)
    b = rng.uniform(-1, 1, (batch, cb, rb)).astype(np.float32)
    c = rng.uniform(-1, 1, (batch, n, m)).astype(np.float32)
    A, B, Cm = _quantize(a, at).cuda(), _quantize(b, bt).cuda(), _quantize(c, ct).cuda()
    c_in = Cm.float().cpu().numpy().astype(np.float64)
    handle.gemm_batched_ex(ta, tb, m, n, k, alpha, A, DT[at], ra, B, DT[bt], rb, beta, Cm, DT[ct], m, compute=comp)
    torch.cuda.synchronize()
    out = Cm.float().cpu().numpy().astype(np.float64)
    af = A.float().cpu().numpy()
    bf = B.float().cpu().numpy()
    if comp == 6:
        af, bf = _tf32(af), _tf32(bf)
    if comp == 5:
        af = torch.from_numpy(af).bfloat16().float().numpy()
        bf = torch.from_numpy(bf).bfloat16().float().numpy()
    for q in range(batch):
        Am = af[q].T.astype(np.float64)  # (rows, cols) math orientation
        Bm = bf[q].T.astype(np.float64)
        opA = Am.T if ta != "N" else Am
        opB = Bm.T if tb != "N" else Bm
        ref = alpha * opA @ opB + beta * c_in[q].T
        err = np.abs(out[q].T - ref)
        scale = np.abs(alpha) * np.abs(opA) @ np.abs(opB) + abs(beta) * np.abs(c_in[q].T) + 1e-30
        assert np.max(err / scale) <= rtol, np.max(err / scale)


def test_gemm_batched_ex_early_exit(handle):
    """k == 0 or alpha == 0: C = beta * C; beta == 1 leaves C untouched; beta == 0 writes zeros."""
    import torch

    rng = np.random.default_rng(1)
    c = rng.standard_normal((2, 8, 12)).astype(np.float32)
    for alpha, beta, k in [(1.0, 0.5, 0), (0.0, 0.0, 4), (0.0, 1.0, 4), (2.0, -1.5, 0)]:
        Cm = torch.from_numpy(c).half().cuda()
        before = Cm.float().cpu().numpy()
        A = torch.zeros((2, max(k, 1), 12), dtype=torch.float16, device="cuda")
        B = torch.zeros((2, 8, max(k, 1)), dtype=torch.float16, device="cuda")
        handle.gemm_batched_ex("N", "N", 12, 8, k, alpha, A, 1, 12, B, 1, max(k, 1), beta, Cm, 1, 12, compute=2)
        torch.cuda.synchronize()
        expect = np.zeros_like(before) if beta == 0.0 else (before * beta).astype(np.float16).astype(np.float32)
        np.testing.assert_allclose(Cm.float().cpu().numpy(), expect, rtol=1e-3, atol=1e-3)


# ---------------------------------------------------------- mixed precision + refinement --

def conditioned_batch(n, batch, cond, seed):
    """A = Q1 diag(s) Q2^T with Q from QR of Gaussian matrices and s log-spaced 1..cond (FP64),
    returned as the FP64 matrices and their FP32 column-major batch."""
    rng = np.random.default_rng(seed)
    s = np.logspace(0, np.log10(cond), n)
    A64 = np.empty((batch, n, n))
    for b in range(batch):
        q1, _ = np.linalg.qr(rng.standard_normal((n, n)))
        q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
        A64[b] = (q1 * s) @ q2.T
    a32 = np.ascontiguousarray(np.transpose(A64, (0, 2, 1))).astype(np.float32)
    return A64, a32


def host_berr(A, X, B):
    """max over columns of ||b - A x||inf / (||A||inf ||x||inf + ||b||inf), FP64."""
    R = B - A @ X
    an = np.abs(A).sum(1).max()
    return max(np.abs(R[:, c]).max() / (an * np.abs(X[:, c]).max() + np.abs(B[:, c]).max()) for c in range(B.shape[1]))


@pytest.mark.parametrize("n,batch,compute,max_iter", [(48, 8, 2, 10), (48, 8, 6, 10), (256, 6, 6, 10),
                                                      (256, 6, 2, 10), (256, 4, 5, 40), (512, 2, 6, 10)])
def test_refine_reaches_fp32_backward_error(handle, n, batch, compute, max_iter):
    """kappa = 1e4, nrhs = 16: the refined solution's backward error against the FP32-stored
    matrix, recomputed on the host in FP64, is <= 1e-6 (the device-reported value agrees)."""
    import torch

    nrhs = 16
    A64, a32 = conditioned_batch(n, batch, 1e4, seed=n + compute)
    b = np.random.default_rng(7).standard_normal((batch, nrhs, n)).astype(np.float32)
    A, B = to_dev(a32, "cuda"), to_dev(b, "cuda")
    X, LU, piv, info, berr, iters = handle.refine(A, B, n, nrhs, compute=compute, max_iter=max_iter, tol=1e-6)
    torch.cuda.synchronize()
    assert int(info.max()) == 0
    x = to_host(X)
    dev_berr = to_host(berr)
    it = to_host(iters)
    assert np.all(it < max_iter), it
    for q in range(batch):
        Aq = a32[q].T.astype(np.float64)  # the FP32 matrix the solver saw
        e = host_berr(Aq, x[q].T.astype(np.float64), b[q].T.astype(np.float64))
        assert e <= 1e-6, (q, e)
        assert abs(e - dev_berr[q]) <= 1e-9 + 1e-3 * e
    # the unchanged inputs
    assert np.array_equal(to_host(A), a32) and np.array_equal(to_host(B), b)


def test_refine_plain_factors_match_getrf(handle):
    """With ACLBLAS_COMPUTE_32F the factorisation inside the refinement call is the plain path."""
    import torch

    n, batch = 40, 5
    _, a32 = conditioned_batch(n, batch, 1e2, seed=3)
    b = np.random.default_rng(4).standard_normal((batch, 2, n)).astype(np.float32)
    X, LU, piv, info, berr, iters = handle.refine(to_dev(a32, "cuda"), to_dev(b, "cuda"), n, 2, compute=2,
                                                  max_iter=3)
    torch.cuda.synchronize()
    olu = a32.copy()
    opiv, oinfo, _ = O.port_getrf(olu, n, n)
    np.testing.assert_array_equal(to_host(piv), opiv)
    assert np.array_equal(to_host(LU).view(np.uint32), olu.view(np.uint32))


# --------------------------------------------------------------------------- adjoint --

def _adjoint_inputs(n, nrhs, batch, seed):
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((batch, n, n)) + 8.0 * np.eye(n)
    a32 = np.ascontiguousarray(np.transpose(G, (0, 2, 1))).astype(np.float32)
    b = rng.standard_normal((batch, nrhs, n)).astype(np.float32)
    dx = rng.standard_normal((batch, nrhs, n)).astype(np.float32)
    return a32, b, dx


@pytest.mark.parametrize("n,nrhs", [(64, 8), (16, 3), (32, 1), (100, 5)])
def test_adjoint_matches_fp64_reference_gradient(handle, n, nrhs):
    import torch

    batch = 16
    a32, b, dx = _adjoint_inputs(n, nrhs, batch, seed=n)
    LU = to_dev(a32, "cuda")
    X = to_dev(b, "cuda")
    piv, info = handle.getrf(LU, n, n)
    handle.getrs("N", LU, n, n, piv, X, nrhs, n)
    dB = to_dev(dx, "cuda")
    dA = torch.empty_like(LU)
    handle.adjoint(LU, n, n, piv, X, n, dB, n, dA, n)
    torch.cuda.synchronize()
    for q in range(batch):
        A = a32[q].T.astype(np.float64)
        Xr = np.linalg.solve(A, b[q].T.astype(np.float64))
        dBr = np.linalg.solve(A.T, dx[q].T.astype(np.float64))
        dAr = -dBr @ Xr.T
        assert O.normwise_rel(to_host(dB)[q].T, dBr) <= 1e-4
        assert O.normwise_rel(to_host(dA)[q].T, dAr) <= 1e-4


def test_autograd_solve_gradcheck_fp64_finite_differences(ob, cuda):
    """The autograd Function's analytic gradient (FP32 kernels) against central finite
    differences of the FP64 solve, along random directions, and against the FP64 gradient."""
    import torch

    n, nrhs, batch = 64, 8, 4
    a32, b, dx = _adjoint_inputs(n, nrhs, batch, seed=5)
    A = torch.from_numpy(a32).cuda().requires_grad_(True)
    B = torch.from_numpy(b).cuda().requires_grad_(True)
    W = torch.from_numpy(dx).cuda()
    X = ob.batched_solve(A, B)
    (X * W).sum().backward()
    gA, gB = A.grad.double(), B.grad.double()

    def f64(Ad, Bd):  # column-major batch convention -> math orientation
        return (torch.linalg.solve(Ad.transpose(1, 2), Bd.transpose(1, 2)).transpose(1, 2) * W.double()).sum()

    A64, B64 = A.detach().double(), B.detach().double()
    g = torch.Generator(device="cuda").manual_seed(0)
    h = 1e-6
    for _ in range(4):
        EA = torch.randn(A64.shape, device="cuda", dtype=torch.float64, generator=g)
        EB = torch.randn(B64.shape, device="cuda", dtype=torch.float64, generator=g)
        fd = (f64(A64 + h * EA, B64 + h * EB) - f64(A64 - h * EA, B64 - h * EB)) / (2 * h)
        an = (gA * EA).sum() + (gB * EB).sum()
        assert abs(float(an - fd)) <= 1e-4 * max(1.0, abs(float(fd))), (float(an), float(fd))
    # FP64 reference gradient
    Ad = A64.transpose(1, 2)
    Xd = torch.linalg.solve(Ad, B64.transpose(1, 2))
    dBd = torch.linalg.solve(Ad.transpose(1, 2), W.double().transpose(1, 2))
    dAd = -dBd @ Xd.transpose(1, 2)
    assert float((gB.transpose(1, 2) - dBd).norm() / dBd.norm()) <= 1e-4
    assert float((gA.transpose(1, 2) - dAd).norm() / dAd.norm()) <= 1e-4


@pytest.mark.parametrize("compute", [2, 5, 6])
def test_refine_full_occupancy(handle, compute):
    """kappa = 1e4 at a batch that fills every SM several times: every matrix converges to an
    FP64 backward error <= 1e-6 (no matrix left behind by a race)."""
    import torch

    n, batch, nrhs = 192, 1024, 4
    g = torch.Generator(device="cuda").manual_seed(compute)
    q1, _ = torch.linalg.qr(torch.randn(batch, n, n, device="cuda", dtype=torch.float64, generator=g))
    q2, _ = torch.linalg.qr(torch.randn(batch, n, n, device="cuda", dtype=torch.float64, generator=g))
    s = torch.logspace(0, 4, n, device="cuda", dtype=torch.float64)
    A = ((q1 * s) @ q2.transpose(1, 2)).transpose(1, 2).contiguous().float()
    B = torch.randn(batch, nrhs, n, device="cuda", generator=g)
    X, LU, piv, info, berr, iters = handle.refine(A, B, n, nrhs, compute=compute, max_iter=40, tol=1e-6)
    torch.cuda.synchronize()
    a64 = A.double().transpose(1, 2)
    x64 = X.double().transpose(1, 2)
    b64 = B.double().transpose(1, 2)
    r = b64 - a64 @ x64
    an = a64.abs().sum(2).amax(1)
    e = (r.abs().amax(1) / (an[:, None] * x64.abs().amax(1) + b64.abs().amax(1))).amax(1)
    assert float(e.max()) <= 1e-6, float(e.max())
    assert int(iters.max()) < 40


def _apply_pivots(a, piv):
    """Rows of a (n x n, math orientation) interchanged as LAPACK laswp with 1-based pivots."""
    a = a.copy()
    for k, p in enumerate(piv):
        p = int(p) - 1
        if 0 <= p < a.shape[0] and p != k:
            a[[k, p]] = a[[p, k]]
    return a


@pytest.mark.parametrize("compute,rtol", [(6, 2e-6), (5, 1e-4)], ids=["tf32", "bf16"])
@pytest.mark.parametrize("n", [33, 48, 100, 128, 129, 200, 255, 256])
def test_tmem_mixed_lu_reconstructs(handle, n, compute, rtol):
    """TF32 / BF16 modes (factors resident in tensor memory, split hi/lo tcgen05 trailing update):
    the factors reproduce P*A = L*U in FP64 to the split's precision, pivots form a permutation,
    and refinement reaches an FP64 backward error <= 1e-6."""
    import torch

    batch, nrhs = 12, 2
    A64, a32 = conditioned_batch(n, batch, 1e3, seed=n)
    b = np.random.default_rng(n).standard_normal((batch, nrhs, n)).astype(np.float32)
    X, LU, piv, info, berr, iters = handle.refine(to_dev(a32, "cuda"), to_dev(b, "cuda"), n, nrhs,
                                                  compute=compute, max_iter=10, tol=1e-6)
    torch.cuda.synchronize()
    assert int(info.max()) == 0 and int(info.min()) == 0
    lu, pv = to_host(LU), to_host(piv)
    for q in range(batch):
        assert sorted(_apply_pivots(np.arange(n)[:, None].astype(float), pv[q])[:, 0].astype(int)) == list(range(n))
        F = lu[q].T.astype(np.float64)
        L = np.tril(F, -1) + np.eye(n)
        U = np.triu(F)
        PA = _apply_pivots(a32[q].T.astype(np.float64), pv[q])
        rel = np.linalg.norm(PA - L @ U) / np.linalg.norm(PA)
        assert rel < rtol, (q, rel)
    assert float(to_host(berr).max()) <= 1e-6


@pytest.mark.parametrize("compute", [6, 5], ids=["tf32", "bf16"])
def test_tmem_mixed_lu_singular(handle, compute):
    """A zero column stops the mixed-mode factorisation with info = that column + 1."""
    import torch

    n, batch = 96, 4
    rng = np.random.default_rng(9)
    a = rng.standard_normal((batch, n, n)).astype(np.float32)
    for q, col in enumerate([0, 31, 32, 77]):
        a[q, col, :] = 0.0  # column col (column-major batch convention)
    b = rng.standard_normal((batch, 1, n)).astype(np.float32)
    X, LU, piv, info, berr, iters = handle.refine(to_dev(a, "cuda"), to_dev(b, "cuda"), n, 1, compute=compute,
                                                  max_iter=2, tol=1e-6)
    torch.cuda.synchronize()
    inf = to_host(info)
    assert inf[0] == 1 and inf[1] >= 1 and inf[2] >= 1 and inf[3] >= 1
    assert all(i <= c + 1 for i, c in zip(inf, [0, 31, 32, 77]))


@pytest.mark.parametrize("n", [257, 300, 512, 545, 700])
def test_blocked_tc_lu_reconstructs(handle, n):
    """TF32 mode above n = 256 (blocked LU: FP32 panels, split-TF32 tcgen05 trailing updates fed
    by TMA, row interchanges folded into the update's reads): P*A = L*U in FP64 to the split's
    precision, the pivots form a permutation, and refinement reaches an FP64 backward error <= 1e-6.
    545 and 700 factor their first panels with 1024-thread CTAs; 300 and 545 end on a partial panel."""
    import torch

    batch, nrhs = 3, 2
    A64, a32 = conditioned_batch(n, batch, 1e3, seed=n)
    b = np.random.default_rng(n).standard_normal((batch, nrhs, n)).astype(np.float32)
    X, LU, piv, info, berr, iters = handle.refine(to_dev(a32, "cuda"), to_dev(b, "cuda"), n, nrhs,
                                                  compute=6, max_iter=10, tol=1e-6)
    torch.cuda.synchronize()
    assert int(info.max()) == 0 and int(info.min()) == 0
    lu, pv = to_host(LU), to_host(piv)
    for q in range(batch):
        assert sorted(_apply_pivots(np.arange(n)[:, None].astype(float), pv[q])[:, 0].astype(int)) == list(range(n))
        F = lu[q].T.astype(np.float64)
        L = np.tril(F, -1) + np.eye(n)
        U = np.triu(F)
        PA = _apply_pivots(a32[q].T.astype(np.float64), pv[q])
        rel = np.linalg.norm(PA - L @ U) / np.linalg.norm(PA)
        assert rel < 3e-6, (q, rel)
    assert float(to_host(berr).max()) <= 1e-6
    st, flags = handle.device_status()
    assert st == 0 and flags == 0


def test_blocked_tc_lu_singular(handle):
    """A zero column stops the blocked factorisation with info <= that column + 1; the other
    matrices of the batch are factored and refined as usual."""
    import torch

    n, batch, nrhs = 320, 4, 1
    A64, a32 = conditioned_batch(n, batch, 1e2, seed=3)
    for q, col in enumerate([0, 40, 300]):
        a32[q, col, :] = 0.0
    b = np.random.default_rng(5).standard_normal((batch, nrhs, n)).astype(np.float32)
    X, LU, piv, info, berr, iters = handle.refine(to_dev(a32, "cuda"), to_dev(b, "cuda"), n, nrhs, compute=6,
                                                  max_iter=5, tol=1e-6)
    torch.cuda.synchronize()
    inf = to_host(info)
    assert inf[0] == 1 and 1 <= inf[1] <= 41 and 1 <= inf[2] <= 301
    assert inf[3] == 0 and float(to_host(berr)[3]) <= 1e-6


def test_blocked_tc_lu_full_occupancy(handle):
    """n = 512 at the benchmark's kappa = 1e4, 300 matrices (two waves of panel CTAs): every matrix
    converges to an FP64 backward error <= 1e-6."""
    import torch

    n, batch, nrhs = 512, 300, 4
    g = torch.Generator(device="cuda").manual_seed(11)
    q1, _ = torch.linalg.qr(torch.randn(batch, n, n, device="cuda", dtype=torch.float64, generator=g))
    q2, _ = torch.linalg.qr(torch.randn(batch, n, n, device="cuda", dtype=torch.float64, generator=g))
    s = torch.logspace(0, 4, n, device="cuda", dtype=torch.float64)
    A = ((q1 * s) @ q2.transpose(1, 2)).transpose(1, 2).contiguous().float()
    del q1, q2
    B = torch.randn(batch, nrhs, n, device="cuda", generator=g)
    X, LU, piv, info, berr, iters = handle.refine(A, B, n, nrhs, compute=6, max_iter=10, tol=1e-6)
    torch.cuda.synchronize()
    assert int(info.abs().max()) == 0
    a64 = A.double().transpose(1, 2)
    x64 = X.double().transpose(1, 2)
    b64 = B.double().transpose(1, 2)
    r = b64 - a64 @ x64
    an = a64.abs().sum(2).amax(1)
    e = (r.abs().amax(1) / (an[:, None] * x64.abs().amax(1) + b64.abs().amax(1))).amax(1)
    assert float(e.max()) <= 1e-6, float(e.max())
