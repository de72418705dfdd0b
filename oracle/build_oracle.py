"""Build recipe for the CPU checkers -- test infrastructure only.

* ``oracle/lib/liboracle.so``: this project's C restatement of the reference kernels
  (``lu_oracle.c``) and of the reference's test-input generators (``case_inputs.cpp``).
* ``oracle/_ref/librefgold.so``: the reference's own CPU golden headers, compiled where they
  lie in the reference tree (``refgold.cpp``), linked at run time against scipy's OpenBLAS.
  Built only where the reference tree is present; the built file travels with the repository
  snapshot, the reference sources do not.

Run ``python oracle/build_oracle.py`` or call :func:`build_all`.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
REF_DIR = os.path.join(HERE, "_ref")
ORACLE_LIB = os.path.join(LIB_DIR, "liboracle.so")
REF_LIB = os.path.join(REF_DIR, "librefgold.so")
# The reference tree: OPSBLAS_REFERENCE_ROOT, else a checkout named "reference" beside this repository.
REFERENCE_ROOT = os.environ.get("OPSBLAS_REFERENCE_ROOT",
                                os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference")))


def _openblas_path() -> str:
    import scipy  # noqa: F401  (only to locate scipy.libs)

    libs = glob.glob(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs",
                                  "libscipy_openblas*.so"))
    if not libs:
        raise RuntimeError("scipy's bundled OpenBLAS was not found")
    return libs[0]


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(HERE, "lu_oracle.c"), os.path.join(HERE, "case_inputs.cpp")]
    if not force and not _stale(ORACLE_LIB, srcs):
        return ORACLE_LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    obj = os.path.join(LIB_DIR, "lu_oracle.o")
    # -ffp-contract=off: the only fused multiply-adds are the explicit fmaf() calls.
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-c", srcs[0], "-o", obj])
    subprocess.check_call(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-o", ORACLE_LIB, obj, srcs[1], "-lm"])
    os.remove(obj)
    return ORACLE_LIB


def build_ref(force: bool = False) -> str | None:
    """Compile the reference's golden headers in place; None when the reference is absent."""
    hdrs = [
        os.path.join(REFERENCE_ROOT, "test/getrf_batched/sgetrf_batched/sgetrf_batched_golden.h"),
        os.path.join(REFERENCE_ROOT, "test/getrs_batched/sgetrs_batched_golden.h"),
        os.path.join(REFERENCE_ROOT, "test/getri_batched/sgetri_batched/sgetri_batched_golden.h"),
        os.path.join(REFERENCE_ROOT, "test/geqrf_batched/sgeqrf_batched/sgeqrf_batched_golden.h"),
        os.path.join(REFERENCE_ROOT, "test/gels_batched/sgels_batched/sgels_batched_golden.h"),
    ]
    if not all(os.path.exists(h) for h in hdrs):
        return REF_LIB if os.path.exists(REF_LIB) else None
    src = os.path.join(HERE, "refgold.cpp")
    if not force and not _stale(REF_LIB, [src] + hdrs):
        return REF_LIB
    os.makedirs(REF_DIR, exist_ok=True)
    cmd = [
        "g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-fopenmp",
        f'-DOPENBLAS_DEFAULT_PATH="{_openblas_path()}"',
        "-I", os.path.join(REFERENCE_ROOT, "include"),
        "-I", os.path.join(HERE, "ref_stub"),
        "-I", os.path.dirname(hdrs[0]),
        "-I", os.path.dirname(hdrs[1]),
        "-I", os.path.dirname(hdrs[2]),
        "-I", os.path.dirname(hdrs[3]),
        "-I", os.path.dirname(hdrs[4]),
        "-o", REF_LIB, src, "-ldl",
    ]
    subprocess.check_call(cmd)
    return REF_LIB


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_LIB, os.path.exists(ORACLE_LIB))
    print(REF_LIB, os.path.exists(REF_LIB))
