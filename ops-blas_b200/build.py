"""Build libopsblas_b200.so (sm_100a) in-tree with nvcc.

Every ``csrc/*.cu`` file is compiled to an object in ``_build/`` (in parallel), then linked
into ``libopsblas_b200.so`` next to this file with the CUDA runtime linked statically, so the
library loads in any process regardless of which CUDA runtime that process already uses.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libopsblas_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I", INCLUDE, "-I", CSRC,
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "acl", "*.h")))


def _obj(src: str) -> str:
    return os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")


def _compile(src: str, extra: list[str]) -> str:
    obj = _obj(src)
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose_ptxas: bool = False, jobs: int | None = None) -> str:
    """Compile what changed and relink; returns the library path."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    hdr_mtime = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    todo = [s for s in srcs if force or not os.path.exists(_obj(s))
            or os.path.getmtime(_obj(s)) < max(os.path.getmtime(s), hdr_mtime)]
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for src, log in zip(todo, ex.map(lambda s: _compile(s, extra), todo)):
                if verbose_ptxas and log:
                    sys.stderr.write(f"== {os.path.basename(src)}\n{log}")
    objs = [_obj(s) for s in srcs]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", tmp, *objs]
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
