"""Helpers for the GPU parity tests: build the CUDA-path objects for a golden case."""
from __future__ import annotations

import copy

import numpy as np
import torch

from conftest import golden_setup


def make_equation(case, solver_name="Butcher", solver_extra="RK4", dt=None, cfl=None, state0=None,
                  **cfg_overrides):
    """(fixture, FVMEquation on cuda, FVMTables, cfg) of a golden case; ``cfg_overrides`` set
    config fields (e.g. ``lim_p``) for both the tables and the equation."""
    from fvm_solver_b200 import equation as E, mesh_store as ms
    g, spec, tables, cfg = golden_setup(case, **cfg_overrides)
    cfg = copy.deepcopy(cfg)
    cfg.device = "cuda"
    cfg.solver_name, cfg.solver_extra = solver_name, solver_extra
    cfg.dt = float(g["dt"]) if dt is None else dt
    cfg.cfl = cfl
    dim = int(g["dim"])
    phy = E.FluidConstitution2D(cfg) if dim == 2 else E.FluidConstitution3D(cfg)
    bc = {} if case == "ptile" else ms.default_bc_tags(spec.bc_tags, dim)
    eq = E.FVMEquation(cfg, phy, spec, dim + 2, bc,
                       us_init=torch.from_numpy(g["state0"]) if state0 is None else state0)
    return g, eq, tables, cfg


def to_np(t):
    return t.detach().cpu().numpy().astype(np.float64)
