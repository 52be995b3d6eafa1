"""Build recipe for the CUDA library ``libfvm_b200.so`` (nvcc, sm_100a, in-tree).

``python -m fvm_solver_b200.build`` compiles ``csrc/*.cu`` into ``fvm_solver_b200/libfvm_b200.so``.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libfvm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def build(verbose: bool = False, extra=()) -> str:
    """Compile (if any source or header is newer than the library) and return the library path."""
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "fvm_b200.h")]
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps) and not extra:
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-Xcompiler", "-fPIC", "-O3", "-std=c++17", "-lineinfo", *ARCH,
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(HERE, "csrc"),
           *extra, *sources(), "-o", tmp, "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
