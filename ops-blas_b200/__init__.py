"""Host-side binding of libopsblas_b200.so, the B200 build of ops-blas's batched LU chain.

The library is a C ABI (``include/cann_ops_blas.h``). This module loads it with ctypes and
offers two layers:

* ``lib()``: the raw C functions with their argtypes (``aclblasSgetrfBatched`` etc.), taking
  device pointers as Python ints, exactly as a C caller would.
* ``Handle`` and the ``*_batched`` helpers: the same calls on torch tensors. A batch is a
  C-contiguous float32 CUDA tensor of shape ``(batch, ncols, ld)``; element (i, j) of matrix b
  is ``t[b, j, i]`` (column-major with leading dimension ``ld``). The helpers build the device
  pointer arrays the C API takes and pass the current torch stream.

There is no fallback: if the shared library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libopsblas_b200.so")

# aclblasStatus_t (include/cann_ops_blas_common.h)
STATUS = {
    0: "SUCCESS", 1: "NOT_INITIALIZED", 2: "ALLOC_FAILED", 3: "INVALID_VALUE", 4: "MAPPING_ERROR",
    5: "EXECUTION_FAILED", 6: "INTERNAL_ERROR", 7: "NOT_SUPPORTED", 8: "ARCH_MISMATCH", 9: "HANDLE_IS_NULLPTR",
    10: "INVALID_ENUM", 11: "UNKNOWN",
}
SUCCESS, NOT_INITIALIZED, ALLOC_FAILED, INVALID_VALUE = 0, 1, 2, 3
EXECUTION_FAILED, INTERNAL_ERROR, NOT_SUPPORTED, ARCH_MISMATCH = 5, 6, 7, 8
HANDLE_IS_NULLPTR, INVALID_ENUM = 9, 10
OP_N, OP_T, OP_C = 111, 112, 113
TRANS = {"N": OP_N, "T": OP_T, "C": OP_C}

_vp = C.c_void_p
_ip = C.POINTER(C.c_int)

# name -> (restype, argtypes); every symbol declared in include/cann_ops_blas.h
SIGNATURES = {
    "aclblasCreate": (C.c_int, [C.POINTER(_vp)]),
    "aclblasDestroy": (C.c_int, [_vp]),
    "aclblasSetStream": (C.c_int, [_vp, _vp]),
    "aclblasGetStream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "aclblasSetWorkspace": (C.c_int, [_vp, _vp, C.c_size_t]),
    "aclblasGetVersion": (C.c_int, [_vp, _ip]),
    "aclblasLoggerConfigure": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_char_p]),
    "aclblasSetLoggerCallback": (C.c_int, [_vp]),
    "aclblasGetLoggerCallback": (C.c_int, [C.POINTER(_vp)]),
    "aclblasGetDeviceStatus": (C.c_int, [_vp, C.POINTER(C.c_uint)]),
    "aclblasSgetrfBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int]),
    "aclblasSgetrsBatched": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _ip,
                                       C.c_int]),
    "aclblasSgetriBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int]),
    "aclblasSmatinvBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, C.c_int]),
    "aclblasSgeqrfBatched": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int]),
    "aclblasBuildPointerArray": (C.c_int, [_vp, _vp, C.c_longlong, C.c_int, _vp]),
    "aclblasSgetrfStridedBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_longlong, _vp, _vp, C.c_int]),
    "aclblasSgetrsStridedBatched": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, C.c_longlong, _vp, _vp,
                                              C.c_int, C.c_longlong, _vp, C.c_int]),
    "aclblasSgetriStridedBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_longlong, _vp, _vp, C.c_int,
                                              C.c_longlong, _vp, C.c_int]),
    "aclblasSgelsBatched": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp,
                                      C.c_int]),
    "aclblasSgemmBatched": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, _vp,
                                      C.c_int, _vp, _vp, C.c_int, C.c_int]),
    "aclblasCgemmBatched": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, _vp,
                                      C.c_int, _vp, _vp, C.c_int, C.c_int]),
    "aclblasGemmBatchedEx": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, C.c_int,
                                       _vp, C.c_int, C.c_int, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "aclblasSgetrfsRefineBatchedEx": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _vp,
                                                C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_double, _vp, _vp,
                                                _vp, C.c_int]),
    "aclblasSgetrfsRefineBatchedStaticScratch": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp,
                                                           _vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_double,
                                                           _vp, _vp, _vp, C.c_int]),
    "aclblasSgetrfGetrsGroupedPlanCreate": (C.c_int, [_vp, C.c_int, _ip, _ip, _ip, _ip, _ip, _ip,
                                                      C.POINTER(_vp)]),
    "aclblasSgetrfGetrsGroupedPlanGetConfig": (C.c_int, [_vp, _ip]),
    "aclblasSgetrfGetrsGroupedPlanDestroy": (C.c_int, [_vp]),
    "aclblasSgetrfGetrsGroupedBatched": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "aclblasSgetrsAdjointBatched": (C.c_int, [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _vp,
                                              C.c_int, _vp, C.c_int, C.c_int]),
}

# aclDataType (include/acl/acl.h) and aclblasComputeType_t (include/cann_ops_blas_common.h)
ACL_FLOAT, ACL_FLOAT16, ACL_BF16, ACL_FLOAT8_E5M2, ACL_FLOAT8_E4M3FN = 0, 1, 27, 35, 36
COMPUTE_16F, COMPUTE_32F, COMPUTE_32F_PEDANTIC, COMPUTE_32F_FAST_16BF, COMPUTE_32F_FAST_TF32 = 0, 2, 3, 5, 6

_lib = None


class AclblasError(RuntimeError):
    def __init__(self, api, status):
        super().__init__(f"{api} returned ACLBLAS_STATUS_{STATUS.get(status, status)} ({status})")
        self.status = status


def lib():
    """The loaded C library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with ops-blas_b200/build.py "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(api, status):
    if status != SUCCESS:
        raise AclblasError(api, status)


# ------------------------------------------------------------------------- torch helpers --

def _torch():
    import torch

    return torch


def ptr_array(t, stride_elems=None, count=None):
    """Device int64 tensor of the addresses of the matrices of batch tensor ``t``."""
    torch = _torch()
    count = t.shape[0] if count is None else count
    stride = (t.stride(0) if stride_elems is None else stride_elems) * t.element_size()
    return (torch.arange(count, device=t.device, dtype=torch.int64) * stride + t.data_ptr()).contiguous()


def _addr(x):
    return None if x is None else x.data_ptr()


class Handle:
    """aclblasHandle_t bound to the current torch stream at creation (re-bind with set_stream)."""

    def __init__(self, stream=None):
        self._ws = None
        self.h = _vp()
        check("aclblasCreate", lib().aclblasCreate(C.byref(self.h)))
        self.set_stream(stream)

    def set_stream(self, stream=None):
        torch = _torch()
        s = torch.cuda.current_stream() if stream is None else stream
        check("aclblasSetStream", lib().aclblasSetStream(self.h, _vp(s.cuda_stream)))
        self.stream = s

    def device_status(self):
        """(status, flags) of aclblasGetDeviceStatus: synchronises the handle's stream, returns
        the bits that kernels set when a bounded wait gave up (and clears them)."""
        flags = C.c_uint(0)
        st = lib().aclblasGetDeviceStatus(self.h, C.byref(flags))
        return st, flags.value

    def close(self):
        if self.h:
            check("aclblasDestroy", lib().aclblasDestroy(self.h))
            self.h = _vp()
        self._ws = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- batched LU chain on torch tensors ------------------------------------------------

    def getrf(self, A, n, lda, piv=None, info=None, pivot=True, aptr=None):
        """In-place LU of every matrix of A (batch, n, lda); returns (piv, info) int32 tensors."""
        torch = _torch()
        batch = A.shape[0]
        if pivot and piv is None:
            piv = torch.empty((batch, max(1, n)), dtype=torch.int32, device=A.device)
        if info is None:
            info = torch.empty(batch, dtype=torch.int32, device=A.device)
        aptr = ptr_array(A) if aptr is None else aptr
        check("aclblasSgetrfBatched", lib().aclblasSgetrfBatched(
            self.h, n, aptr.data_ptr(), lda, _addr(piv) if pivot else None, info.data_ptr(), batch))
        return (piv if pivot else None), info

    def getrs(self, trans, LU, n, lda, piv, B, nrhs, ldb, aptr=None, bptr=None):
        """In-place solve op(A) X = B; trans in 'N', 'T', 'C'. Returns the host info value."""
        info = C.c_int(-7)
        aptr = ptr_array(LU) if aptr is None else aptr
        bptr = ptr_array(B) if bptr is None else bptr
        check("aclblasSgetrsBatched", lib().aclblasSgetrsBatched(
            self.h, TRANS[trans], n, nrhs, aptr.data_ptr(), lda, _addr(piv), bptr.data_ptr(), ldb,
            C.byref(info), LU.shape[0]))
        return info.value

    def gemm_batched_ex(self, transa, transb, m, n, k, alpha, A, atype, lda, B, btype, ldb, beta, Cm, ctype, ldc,
                        compute=COMPUTE_32F, aptr=None, bptr=None, cptr=None):
        """aclblasGemmBatchedEx on batch tensors; alpha/beta are Python floats."""
        a = C.c_float(alpha)
        b = C.c_float(beta)
        aptr = ptr_array(A) if aptr is None else aptr
        bptr = ptr_array(B) if bptr is None else bptr
        cptr = ptr_array(Cm) if cptr is None else cptr
        check("aclblasGemmBatchedEx", lib().aclblasGemmBatchedEx(
            self.h, TRANS[transa], TRANS[transb], m, n, k, C.byref(a), aptr.data_ptr(), atype, lda,
            bptr.data_ptr(), btype, ldb, C.byref(b), cptr.data_ptr(), ctype, ldc, Cm.shape[0], compute, 0))

    def refine(self, A, B, n, nrhs, compute=COMPUTE_32F_FAST_TF32, max_iter=10, tol=1e-6):
        """Factor + solve + iterative refinement (aclblasSgetrfsRefineBatchedEx).
        A (batch, n, n) and B (batch, nrhs, n) are left unchanged. Returns
        (X, LU, piv, info, berr, iters)."""
        torch = _torch()
        batch = A.shape[0]
        dev = A.device
        LU = torch.empty_like(A)
        X = torch.empty_like(B)
        piv = torch.empty((batch, n), dtype=torch.int32, device=dev)
        info = torch.empty(batch, dtype=torch.int32, device=dev)
        berr = torch.empty(batch, dtype=torch.float64, device=dev)
        iters = torch.empty(batch, dtype=torch.int32, device=dev)
        need = (((n * nrhs * 4 + 255) // 256) * 256 + 20) * batch + 512
        if 256 < n <= 1024:  # scratch of the blocked tensor-core LU (TF32 mode), after the refinement's part
            plane = (n - 32) * 32 * 4
            per = 2 * ((2 * plane + 255) // 256 * 256)
            need = (need + 255) // 256 * 256 + per * batch + batch * 16 + 512
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(max(need, 32 << 20), dtype=torch.uint8, device=dev)
            check("aclblasSetWorkspace", lib().aclblasSetWorkspace(self.h, _vp(self._ws.data_ptr()),
                                                                   self._ws.numel()))
        # the pointer arrays must stay referenced until the call has been enqueued: a temporary
        # freed inside the argument list would hand its memory to the next one
        pa, plu, pb, px = ptr_array(A), ptr_array(LU), ptr_array(B), ptr_array(X)
        check("aclblasSgetrfsRefineBatchedEx", lib().aclblasSgetrfsRefineBatchedEx(
            self.h, n, nrhs, pa.data_ptr(), n, plu.data_ptr(), n, piv.data_ptr(), pb.data_ptr(), n, px.data_ptr(), n,
            compute, max_iter, tol, berr.data_ptr(), iters.data_ptr(), info.data_ptr(), batch))
        return X, LU, piv, info, berr, iters

    def adjoint(self, LU, n, lda, piv, X, ldx, dX, lddx, dA=None, ldda=None):
        """dX <- A^{-T} dX (= dB); dA <- -dB X^T when dA is given (aclblasSgetrsAdjointBatched)."""
        nrhs = X.shape[1]
        plu, px, pdx = ptr_array(LU), ptr_array(X), ptr_array(dX)
        pda = None if dA is None else ptr_array(dA)
        check("aclblasSgetrsAdjointBatched", lib().aclblasSgetrsAdjointBatched(
            self.h, n, nrhs, plu.data_ptr(), lda, _addr(piv), px.data_ptr(), ldx, pdx.data_ptr(), lddx,
            None if pda is None else pda.data_ptr(), ldda if ldda is not None else n, LU.shape[0]))

    def getri(self, LU, n, lda, piv, Cinv, ldc, info=None, aptr=None, cptr=None):
        """Cinv = inverse from the LU factors; returns the info tensor."""
        torch = _torch()
        if info is None:
            info = torch.empty(LU.shape[0], dtype=torch.int32, device=LU.device)
        aptr = ptr_array(LU) if aptr is None else aptr
        cptr = ptr_array(Cinv) if cptr is None else cptr
        check("aclblasSgetriBatched", lib().aclblasSgetriBatched(
            self.h, n, aptr.data_ptr(), lda, _addr(piv), cptr.data_ptr(), ldc, info.data_ptr(), LU.shape[0]))
        return info

    def sgemm(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, aptr=None, bptr=None,
              cptr=None):
        """aclblasSgemmBatched over batch tensors A, B, C (column-major matrices); alpha, beta floats."""
        aptr = ptr_array(A) if aptr is None else aptr
        bptr = ptr_array(B) if bptr is None else bptr
        cptr = ptr_array(Cm) if cptr is None else cptr
        al, be = C.c_float(alpha), C.c_float(beta)
        check("aclblasSgemmBatched", lib().aclblasSgemmBatched(
            self.h, TRANS[transa], TRANS[transb], m, n, k, C.byref(al), aptr.data_ptr(), lda, bptr.data_ptr(), ldb,
            C.byref(be), cptr.data_ptr(), ldc, Cm.shape[0]))

    def cgemm(self, transa, transb, m, n, k, alpha, A, lda, B, ldb, beta, Cm, ldc, aptr=None, bptr=None,
              cptr=None):
        """aclblasCgemmBatched over complex64 batch tensors A, B, C (column-major matrices);
        alpha, beta Python complex values (aclblasComplex: real, then imaginary)."""
        aptr = ptr_array(A) if aptr is None else aptr
        bptr = ptr_array(B) if bptr is None else bptr
        cptr = ptr_array(Cm) if cptr is None else cptr
        al = (C.c_float * 2)(complex(alpha).real, complex(alpha).imag)
        be = (C.c_float * 2)(complex(beta).real, complex(beta).imag)
        check("aclblasCgemmBatched", lib().aclblasCgemmBatched(
            self.h, TRANS[transa], TRANS[transb], m, n, k, al, aptr.data_ptr(), lda, bptr.data_ptr(), ldb,
            be, cptr.data_ptr(), ldc, cptr.shape[0]))

    def geqrf(self, A, m, n, lda, tau=None, aptr=None, tptr=None):
        """In-place QR of every matrix of A (batch, n, lda); returns the tau tensor (batch, min(m,n))."""
        torch = _torch()
        if tau is None:
            tau = torch.zeros((A.shape[0], max(1, min(m, n))), dtype=torch.float32, device=A.device)
        aptr = ptr_array(A) if aptr is None else aptr
        tptr = ptr_array(tau) if tptr is None else tptr
        info = C.c_int(-99)
        check("aclblasSgeqrfBatched", lib().aclblasSgeqrfBatched(
            self.h, m, n, aptr.data_ptr(), lda, tptr.data_ptr(), C.byref(info), A.shape[0]))
        assert info.value == 0, info.value
        return tau

    def gels(self, trans, A, m, n, nrhs, lda, Cm, ldc, info=None, aptr=None, cptr=None):
        """aclblasSgelsBatched in place on batch tensors A (batch, n, lda) and C (batch, nrhs, ldc);
        returns the per-matrix info tensor."""
        torch = _torch()
        if info is None:
            info = torch.full((A.shape[0],), -1, dtype=torch.int32, device=A.device)
        aptr = ptr_array(A) if aptr is None else aptr
        cptr = ptr_array(Cm) if cptr is None else cptr
        check("aclblasSgelsBatched", lib().aclblasSgelsBatched(
            self.h, TRANS[trans], m, n, nrhs, aptr.data_ptr(), lda, cptr.data_ptr(), ldc, info.data_ptr(),
            A.shape[0]))
        return info

    def matinv(self, A, n, lda, Ainv, lda_inv, info=None, aptr=None, cptr=None):
        """Ainv = inverse of every matrix of A (n <= 32) in one launch; returns the info tensor."""
        torch = _torch()
        if info is None:
            info = torch.empty(A.shape[0], dtype=torch.int32, device=A.device)
        aptr = ptr_array(A) if aptr is None else aptr
        cptr = ptr_array(Ainv) if cptr is None else cptr
        check("aclblasSmatinvBatched", lib().aclblasSmatinvBatched(
            self.h, n, aptr.data_ptr(), lda, cptr.data_ptr(), lda_inv, info.data_ptr(), A.shape[0]))
        return info


# ------------------------------------------------------------------- grouped factor+solve --

def _int_array(vals):
    vals = [int(v) for v in vals]
    return (C.c_int * max(len(vals), 1))(*vals)


class GroupedPlan:
    """aclblasGroupedPlan_t for groups of instances sharing (n, nrhs, lda, ldb).

    ``ns``, ``nrhss``, ``sizes`` (and optionally ``ldas``, ``ldbs``, default n) are per group;
    ``config`` is None or one (lanes, warps, panel) triple per group, 0 = the tuning table's
    choice. Instances are numbered group by group."""

    def __init__(self, handle, ns, nrhss, sizes, ldas=None, ldbs=None, config=None):
        self.ns = [int(v) for v in ns]
        self.nrhss = [int(v) for v in nrhss]
        self.sizes = [int(v) for v in sizes]
        self.ldas = [max(1, v) for v in self.ns] if ldas is None else [int(v) for v in ldas]
        self.ldbs = [max(1, v) for v in self.ns] if ldbs is None else [int(v) for v in ldbs]
        cfg = None if config is None else _int_array([x for t in config for x in t])
        self.p = _vp()
        check("aclblasSgetrfGetrsGroupedPlanCreate", lib().aclblasSgetrfGetrsGroupedPlanCreate(
            handle.h, len(self.ns), _int_array(self.ns), _int_array(self.nrhss), _int_array(self.ldas),
            _int_array(self.ldbs), _int_array(self.sizes), cfg, C.byref(self.p)))

    def config(self):
        out = (C.c_int * max(3 * len(self.ns), 1))()
        check("aclblasSgetrfGetrsGroupedPlanGetConfig", lib().aclblasSgetrfGetrsGroupedPlanGetConfig(self.p, out))
        return [tuple(out[3 * g:3 * g + 3]) for g in range(len(self.ns))]

    def run(self, handle, aptr, piv, info, bptr=None):
        """Executes the plan: aptr / bptr are device pointer arrays (int64 tensors) in instance
        order, piv the concatenated pivots, info one int per instance."""
        check("aclblasSgetrfGetrsGroupedBatched", lib().aclblasSgetrfGetrsGroupedBatched(
            handle.h, self.p, aptr.data_ptr(), piv.data_ptr(), info.data_ptr(),
            None if bptr is None else bptr.data_ptr()))

    def close(self):
        if self.p:
            check("aclblasSgetrfGetrsGroupedPlanDestroy", lib().aclblasSgetrfGetrsGroupedPlanDestroy(self.p))
            self.p = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grouped_offsets(ns, cols, lds, sizes, align=64):
    """Offsets (in floats) of the instances of a grouped batch packed in one slab: instance i of
    group g takes lds[g] * cols[g] floats, each starting on an ``align``-float boundary.
    Returns (offsets list, total floats)."""
    offs, cur = [], 0
    for n, c, ld, sz in zip(ns, cols, lds, sizes):
        span = ld * c
        for _ in range(sz):
            offs.append(cur)
            cur += (span + align - 1) // align * align
    return offs, max(cur, 1)


def slab_ptrs(slab, offsets):
    """Device int64 tensor of slab.data_ptr() + 4 * offset for each offset."""
    torch = _torch()
    off = torch.tensor(offsets, dtype=torch.int64, device=slab.device)
    return (off * slab.element_size() + slab.data_ptr()).contiguous()


def grouped_plain(handle, ns, nrhss, sizes, ldas, ldbs, aptr, piv, info, bptr=None):
    """The same work as GroupedPlan.run through the plain entry points: per group one
    aclblasSgetrfBatched and one aclblasSgetrsBatched (trans N) on the group's slice of the
    pointer arrays. This is the plain FP32 path the grouped launch is compared with."""
    L = lib()
    first = poff = 0
    info_h = C.c_int(0)
    for n, nrhs, sz, lda, ldb in zip(ns, nrhss, sizes, ldas, ldbs):
        if sz > 0 and n > 0:
            a = aptr.data_ptr() + 8 * first
            p = piv.data_ptr() + 4 * poff
            check("aclblasSgetrfBatched", L.aclblasSgetrfBatched(handle.h, n, a, lda, p, info.data_ptr() + 4 * first,
                                                                 sz))
            if nrhs > 0:
                check("aclblasSgetrsBatched", L.aclblasSgetrsBatched(handle.h, OP_N, n, nrhs, a, lda, p,
                                                                     bptr.data_ptr() + 8 * first, ldb,
                                                                     C.byref(info_h), sz))
        first += sz
        poff += n * sz


# ------------------------------------------------------------------ differentiable solve --

_default_handle = None


def default_handle():
    global _default_handle
    if _default_handle is None:
        _default_handle = Handle()
    else:
        _default_handle.set_stream()
    return _default_handle


def _solve_function():
    torch = _torch()

    class BatchedSolve(torch.autograd.Function):
        """X = A^{-1} B for a batch. A: (batch, n, n), B: (batch, nrhs, n), both in the
        column-major batch convention of this module (element (i, j) of A[b] is A[b, j, i]).
        Forward: getrf + getrs (N). Backward: aclblasSgetrsAdjointBatched on the saved LU
        factors and pivots -- dB = A^{-T} dX, dA = -dB X^T."""

        @staticmethod
        def forward(ctx, A, B):
            h = default_handle()
            n = A.shape[1]
            LU = A.detach().contiguous().clone()
            X = B.detach().contiguous().clone()
            piv, info = h.getrf(LU, n, n)
            h.getrs("N", LU, n, n, piv, X, X.shape[1], n)
            ctx.save_for_backward(LU, piv, X)
            return X

        @staticmethod
        def backward(ctx, dX):
            LU, piv, X = ctx.saved_tensors
            h = default_handle()
            n = LU.shape[1]
            dB = dX.detach().contiguous().clone()
            dA = torch.empty_like(LU) if ctx.needs_input_grad[0] else None
            h.adjoint(LU, n, n, piv, X, n, dB, n, dA, n)
            return dA, (dB if ctx.needs_input_grad[1] else None)

    return BatchedSolve


_BatchedSolve = None


def batched_solve(A, B):
    """Differentiable batched solve through the C ABI (see _solve_function)."""
    global _BatchedSolve
    if _BatchedSolve is None:
        _BatchedSolve = _solve_function()
    return _BatchedSolve.apply(A, B)
