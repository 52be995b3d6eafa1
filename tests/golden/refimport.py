"""Import the reference implementation (Python, CPU path) for fixture generation and checks.

Only the machine that generates the fixtures has the reference sources, named by the environment
variable ``FVM_REFERENCE_PATH`` (the directory that holds ``time_fvm/``); the GPU tests, the smoke
test and the benchmark never import this.
The stubs in ``refstubs/`` stand in for the reference's plotting / coloured-print dependencies,
which are absent here.  ``fp64=True`` applies a dtype shim (default dtype float64 and
``torch.float32`` / ``Tensor.float`` redirected to float64) because the reference hard-codes
float32 in several places; the shim must be applied in a fresh process before the import.
"""
from __future__ import annotations

import os
import sys

REFERENCE_PATH = os.environ.get("FVM_REFERENCE_PATH", "")
_HERE = os.path.dirname(os.path.abspath(__file__))


def reference_available() -> bool:
    """Whether ``FVM_REFERENCE_PATH`` names a checkout of the reference (its ``time_fvm`` package)."""
    return bool(REFERENCE_PATH) and os.path.isdir(os.path.join(REFERENCE_PATH, "time_fvm"))


def import_reference(fp64: bool = False):
    if not reference_available():
        raise RuntimeError("set FVM_REFERENCE_PATH to a checkout of the reference (the directory holding time_fvm/)")
    import torch
    if fp64:
        torch.set_default_dtype(torch.float64)
        torch.float32 = torch.float64
        torch.Tensor.float = torch.Tensor.double
    for p in (os.path.join(_HERE, "refstubs"), REFERENCE_PATH):
        if p not in sys.path:
            sys.path.insert(0, p)
    import importlib
    mods = {}
    for name in ["time_fvm.mesh_utils.fvm_mesh", "time_fvm.mesh_utils.mesh_store",
                 "time_fvm.fvm_equation", "time_fvm.config_fvm", "time_fvm.utils.sparse",
                 "time_fvm.utils.ell_kernel", "time_fvm.time_solvers.integrators",
                 "time_fvm.fvm_stepping.facet_process", "time_fvm.fvm_stepping.facet_boundary"]:
        mods[name.rsplit(".", 1)[1]] = importlib.import_module(name)
    return mods
