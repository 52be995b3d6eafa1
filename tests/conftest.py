"""Shared fixtures: markers, golden-vector loading, host table construction."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def load_golden(case: str) -> dict:
    return dict(np.load(os.path.join(GOLDEN, f"fvm_golden_{case}.npz")))


def golden_setup(case: str, **cfg_overrides):
    """(fixture dict, MeshSpec, FVMTables, cfg) rebuilt from the stored mesh; ``cfg_overrides``
    set config fields (e.g. ``lim_p``) before the tables are built."""
    import torch
    from fvm_solver_b200 import config as cf, fvm_mesh as fm, mesh_store as ms, tables as tb
    from fvm_solver_b200.meshgen import MeshSpec
    g = load_golden(case)
    if case == "ptile":
        return ptile_setup(g, **cfg_overrides)
    dim = int(g["dim"])
    spec = MeshSpec(vertices=torch.from_numpy(g["vertices"]), cells=torch.from_numpy(g["cells"]),
                    facets=torch.from_numpy(g["facets"]),
                    bc_facet_mask=torch.from_numpy(g["bc_facet_mask"]),
                    bc_tags=[str(t) for t in g["bc_tags"]], bound_facets=torch.zeros(0))
    cfg = cf.ConfigEllipse()
    for k, v in cfg_overrides.items():
        setattr(cfg, k, v)
    if dim == 3:
        cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
        cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
    tables = tb.FVMTables(fm.mesh_from_spec(spec), cfg, dim + 2, ms.default_bc_tags(spec.bc_tags, dim))
    return g, spec, tables, cfg


def ptile_setup(g: dict, **cfg_overrides):
    """The periodic Taylor-Green box of the ``ptile`` fixture: its MeshSpec (with lattice shifts),
    the product's periodic tables and the Taylor-Green gas constants the fixture was made with."""
    import torch
    from fvm_solver_b200 import config as cf, fvm_mesh as fm, tables as tb
    from fvm_solver_b200.meshgen import MeshSpec
    spec = MeshSpec(vertices=torch.from_numpy(g["vertices"]), cells=torch.from_numpy(g["cells"]),
                    facets=torch.from_numpy(g["facets"]),
                    bc_facet_mask=torch.zeros(len(g["facets"]), dtype=torch.bool), bc_tags=[],
                    bound_facets=torch.zeros((0, 3), dtype=torch.int64), period=g["period"],
                    cell_shifts=torch.from_numpy(g["cell_shifts"]), facet_shifts=torch.from_numpy(g["facet_shifts"]))
    cfg = cf.TaylorGreenConfig(device="cpu", cfl=None, dt=float(g["dt"]))
    for k, v in cfg_overrides.items():
        setattr(cfg, k, v)
    tables = tb.FVMTables(fm.mesh_from_spec(spec), cfg, 5, {})
    return g, spec, tables, cfg


@pytest.fixture(scope="session", params=["c2d", "b3d"])
def golden(request):
    return golden_setup(request.param)
