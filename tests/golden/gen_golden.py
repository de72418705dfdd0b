"""Generate the golden fixtures of tests/golden/ from the reference's own CPU golden path.

Run where the reference tree is available (it builds oracle/_ref/librefgold.so from the
reference's test golden headers, which call LAPACK through the OpenBLAS bundled with scipy 1.18.1):

    python tests/golden/gen_golden.py

Outputs (compressed .npz, committed):
  c1.npz         -- the parity configuration: n = lda = 16, 1024 matrices, nrhs = 1, A and B
                    i.i.d. N(0,1) from numpy.random.default_rng(0) (A drawn first, then B; no
                    diagonal shift). The inputs are regenerated from the seed (CRC stored); the
                    golden pivots, info and solution X are stored for all 1024 matrices, the
                    golden LU factors for the first 128.
  csv_small.npz  -- golden outputs of the reference's CSV cases with n <= 32 for getrf, getrs
                    and getri (at most the first 4 matrices of a case). Inputs are regenerated
                    by the tests from the reference generators (oracle.case_matrices /
                    case_rhs); a CRC of each input is stored to detect generator drift.
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from cases import GETRF, GETRI, GETRS  # noqa: E402


def crc(a: np.ndarray) -> int:
    return zlib.crc32(np.ascontiguousarray(a).tobytes())


def c1_inputs():
    n, batch = 16, 1024
    rng = np.random.default_rng(0)
    A = rng.standard_normal((batch, n, n)).astype(np.float32)
    B = rng.standard_normal((batch, 1, n)).astype(np.float32)
    return A, B


C1_LU_STORED = 128
MAX_STORED = 4


def keep(case) -> bool:
    return case.status == "SUCCESS" and case.n > 0 and case.batch > 0 and case.n <= 32


def main():
    assert O.ref() is not None, "the reference golden library could not be built (reference tree absent?)"
    out = {}
    A, B = c1_inputs()
    LU = A.copy()
    piv, info = O.ref_getrf(LU, 16, 16, True)
    X = B.copy()
    O.ref_getrs("N", LU, 16, 16, piv, X, 1, 16)
    np.savez_compressed(os.path.join(HERE, "c1.npz"), crcA=np.array(crc(A)), crcB=np.array(crc(B)),
                        LU=LU[:C1_LU_STORED], piv=piv, info=info, X=X,
                        openblas=np.array(O.ref().ref_openblas_config().decode()))

    for c in GETRF:
        if not keep(c):
            continue
        a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
        out[f"getrf/{c.name}/crc"] = np.array(crc(a))
        piv, info = O.ref_getrf(a, c.n, c.lda, c.pivot)
        out[f"getrf/{c.name}/lu"] = a[:MAX_STORED]
        out[f"getrf/{c.name}/info"] = info
        if c.pivot:
            out[f"getrf/{c.name}/piv"] = piv
    for c in GETRS:
        if not keep(c):
            continue
        a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
        b = O.case_rhs(c.n, c.nrhs, c.ldb, c.seed, c.batch)
        out[f"getrs/{c.name}/crc"] = np.array([crc(a), crc(b)])
        piv, info = O.ref_getrf_for_solve(a, c.n, c.lda, c.pivot)
        O.ref_getrs(c.trans, a, c.n, c.lda, piv if c.pivot else None, b, c.nrhs, c.ldb)
        out[f"getrs/{c.name}/x"] = b
        out[f"getrs/{c.name}/rfinfo"] = info
    for c in GETRI:
        if not keep(c):
            continue
        a = O.case_matrices(c.n, c.lda, c.mtype, c.seed, c.batch)
        out[f"getri/{c.name}/crc"] = np.array(crc(a))
        piv, info = O.ref_getrf_for_solve(a, c.n, c.lda, c.pivot)
        cc = np.zeros((c.batch, c.n, c.ldc), np.float32)
        rinfo = O.ref_getri(a, c.n, c.lda, piv if c.pivot else None, cc, c.ldc)
        out[f"getri/{c.name}/c"] = cc[:MAX_STORED]
        out[f"getri/{c.name}/info"] = rinfo
    np.savez_compressed(os.path.join(HERE, "csv_small.npz"), **out)
    for f in ("c1.npz", "csv_small.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
