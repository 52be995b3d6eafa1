"""Degenerate sizes for the persistent kernels (grids of one block, partial warps, tails): tiny
meshes against the FP32 oracle, and the fused step against the separate launches."""
import copy

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(kind):
    from fvm_solver_b200 import config as cf, equation as E, fvm_mesh as fm, meshgen as mg, mesh_store as ms
    from fvm_solver_b200 import tables as tb
    if kind == "box2":
        spec, dim = mg.box3d(2, seed=1), 3
    else:
        spec, dim = mg.channel_cylinder(h=0.25, seed=1, cylinder=False), 2
    cfg = cf.ConfigEllipse()
    if dim == 3:
        cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
        cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
    cfg = copy.deepcopy(cfg)
    cfg.device, cfg.solver_name, cfg.solver_extra, cfg.dt, cfg.cfl = "cuda", "Butcher", "RK4", 1e-4, None
    tags = ms.default_bc_tags(spec.bc_tags, dim)
    T = tb.FVMTables(fm.mesh_from_spec(spec), cfg, dim + 2, tags)
    N = spec.n_cells
    g = torch.Generator().manual_seed(5)
    prim = torch.zeros(N, dim + 2, dtype=torch.float64)
    prim[:, 0] = 3.0 + 0.1 * torch.randn(N, generator=g, dtype=torch.float64)
    prim[:, dim] = 1.0 + 0.01 * torch.randn(N, generator=g, dtype=torch.float64)
    prim[:, dim + 1] = 100.0 + torch.randn(N, generator=g, dtype=torch.float64)
    phy = E.FluidConstitution2D(cfg) if dim == 2 else E.FluidConstitution3D(cfg)
    m, r, Q = phy.primatives_to_state(prim[:, :dim].float(), prim[:, dim:dim + 1].float(), prim[:, dim + 1:].float())
    state = torch.cat([m, r, Q], 1)
    return spec, cfg, tags, T, prim.float(), state, phy, dim


@pytest.mark.parametrize("kind", ["box2", "chan"])
def test_tiny_mesh_vs_oracle(kind):
    from fvm_solver_b200 import equation as E
    from oracle import fvm_oracle as O
    spec, cfg, tags, T, prim, state, phy, dim = _case(kind)
    assert spec.n_cells < 400
    eq = E.FVMEquation(cfg, phy, spec, dim + 2, tags, us_init=state)
    got = eq.forward(prim.cuda()).cpu().numpy()
    want, _ = O.OracleResidual(T, cfg, np.float32).forward(prim.numpy())
    assert rel_l2(got, want) < 1e-5
    eq.reset_gradients()
    eq.t_solver.step(3)
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), state.numpy(), 1e-4)
    for _ in range(3):
        s.butcher_step("RK4")
    assert rel_l2(eq.cells.state.cpu().numpy(), s.state) < 1e-5


@pytest.mark.parametrize("kind", ["box2", "chan"])
def test_tiny_mesh_fused_step(kind):
    from fvm_solver_b200 import equation as E
    spec, cfg, tags, T, prim, state, phy, dim = _case(kind)
    a = E.FVMEquation(cfg, phy, spec, dim + 2, tags, us_init=state)
    b = E.FVMEquation(cfg, phy, spec, dim + 2, tags, us_init=state)
    b.t_solver.fused = True
    a.t_solver.step(4)
    b.t_solver.step(4)
    torch.cuda.synchronize()
    assert torch.equal(a.cells.state, b.cells.state) and b.t_solver.fused_status() == 0
