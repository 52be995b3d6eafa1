"""The C-ABI library: builds, loads without a GPU, exports every function the header declares."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fvm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fvm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    from fvm_solver_b200 import _lib
    from fvm_solver_b200.build import build
    build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert "fvm_residual" in names and "fvm_ell_spmm" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding and vice versa
    assert sorted(_lib.EXPORTED) == names


def test_struct_sizes_match_header():
    """ctypes layouts agree with the C structs (compiled probe of sizeof/offsetof)."""
    import subprocess
    import tempfile
    from fvm_solver_b200 import _lib
    code = r'''
#include <stdio.h>
#include <stddef.h>
#include "fvm_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(fvm_mesh_t), sizeof(fvm_physics_t), sizeof(fvm_work_t),
         sizeof(fvm_tableau_t), sizeof(fvm_solver_bufs_t), offsetof(fvm_mesh_t, ch_vt), offsetof(fvm_tableau_t, cfl));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "p.c")
        open(c, "w").write(code)
        exe = os.path.join(td, "p")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    want = [ctypes.sizeof(_lib.Mesh), ctypes.sizeof(_lib.Physics), ctypes.sizeof(_lib.Work),
            ctypes.sizeof(_lib.Tableau), ctypes.sizeof(_lib.SolverBufs), _lib.Mesh.ch_vt.offset,
            _lib.Tableau.cfl.offset]
    assert [int(x) for x in out] == want


def test_no_cpu_fallback():
    """Without CUDA the product refuses to run instead of silently computing on the CPU."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from fvm_solver_b200 import _lib, sparse
    with pytest.raises(RuntimeError):
        _lib.load()
    A = torch.eye(3).to_sparse()
    with pytest.raises(RuntimeError):
        sparse.to_sparse(A, "cpu")
