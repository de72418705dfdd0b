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
    "aclblasSgetrfBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int]),
    "aclblasSgetrsBatched": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _ip,
                                       C.c_int]),
    "aclblasSgetriBatched": (C.c_int, [_vp, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int]),
}

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
        self.h = _vp()
        check("aclblasCreate", lib().aclblasCreate(C.byref(self.h)))
        self.set_stream(stream)

    def set_stream(self, stream=None):
        torch = _torch()
        s = torch.cuda.current_stream() if stream is None else stream
        check("aclblasSetStream", lib().aclblasSetStream(self.h, _vp(s.cuda_stream)))
        self.stream = s

    def close(self):
        if self.h:
            check("aclblasDestroy", lib().aclblasDestroy(self.h))
            self.h = _vp()

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
