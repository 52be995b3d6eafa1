"""Batched ensemble vs each case run alone (bitwise), and per-case reductions.  Needs a B200."""
import copy

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cases():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    from fvm_solver_b200 import workloads as W
    out = []
    for i, n in enumerate([2100, 3500, 2600, 5200]):
        p = W.ensemble_params(i)
        p["n_cells"] = n
        out.append(W.channel_cylinder(device="cuda", solver_name="AB3", solver_extra="SSP_RK3", cfl=0.3, **p))
    return out


def _run_single(case, cfg, steps):
    eq = case.equation() if cfg is None else None
    if eq is None:
        from fvm_solver_b200.equation import FVMEquation, FluidConstitution2D
        eq = FVMEquation(cfg, FluidConstitution2D(cfg), case.spec, 4, case.bc_tags, us_init=case.state0)
    eq.t_solver.step(steps)
    return eq


@pytest.mark.parametrize("solver", ["AB3", "SSP_RK3"])
def test_batched_equals_single(cases, solver):
    from fvm_solver_b200 import batched as B
    cfgs = []
    for c in cases:
        cfg = copy.deepcopy(c.cfg)
        if solver == "SSP_RK3":
            cfg.solver_name, cfg.solver_extra = "Butcher", "SSP_RK3"
        cfgs.append(cfg)
    parts = []
    for c, cfg in zip(cases, cfgs):
        c2 = copy.copy(c)
        c2.cfg = cfg
        parts.append(B.build_case_tables(c2))
    batch = B.BatchedFVM(parts, cfgs[0], device="cuda")
    batch.t_solver.step(6)
    for k, (c, cfg) in enumerate(zip(cases, cfgs)):
        eq = _run_single(c, cfg, 6)
        assert torch.equal(batch.case_state(k), eq.cells.state), f"case {k}"
        assert torch.equal(batch.t_solver.dt[k:k + 1], eq.t_solver.dt)


def test_batched_graph_and_conservation(cases):
    from fvm_solver_b200 import batched as B
    parts = [B.build_case_tables(c) for c in cases]
    batch = B.BatchedFVM(parts, cases[0].cfg, device="cuda")
    batch.t_solver.track_conservation(True)
    batch.t_solver.step(3)
    replay = batch.t_solver.graph_steps(2)
    replay()
    torch.cuda.synchronize()
    cons = batch.t_solver.cons.cpu().numpy()
    st = batch.cells.state.cpu().double().numpy()
    vol = batch.dev.t.volumes.cpu().numpy()   # uploaded FP64 volumes
    for k in range(len(cases)):
        sl = batch.case_slice(k)
        want = (vol[sl, None] * st[sl]).sum(0)
        assert np.allclose(cons[k], want, rtol=1e-10, atol=1e-8)
    assert torch.isfinite(batch.cells.state).all()


def test_case_mask_freezes_cases(cases):
    """With the case mask, frozen cases keep their state and dt bitwise, and the active ones step
    exactly as without a mask (eager and graph-replayed steps)."""
    from fvm_solver_b200 import batched as B
    parts = [B.build_case_tables(c) for c in cases]
    cfg = copy.deepcopy(cases[0].cfg)
    cfg.solver_name, cfg.solver_extra = "Butcher", "SSP_RK3"
    free = B.BatchedFVM(parts, cfg, device="cuda")
    masked = B.BatchedFVM(parts, cfg, device="cuda")
    start = masked.cells.state.clone()
    dt0 = masked.t_solver.dt.clone()
    masked.use_case_mask(True)
    masked.active.copy_(torch.tensor([1, 0, 1, 0], dtype=torch.uint8))
    free.t_solver.step(2)
    masked.t_solver.step(1)
    masked.t_solver.graph_steps(1)()
    torch.cuda.synchronize()
    for k in range(len(cases)):
        if k in (0, 2):
            assert torch.equal(masked.case_state(k), free.case_state(k)), k
            assert torch.equal(masked.t_solver.dt[k], free.t_solver.dt[k])
        else:
            assert torch.equal(masked.case_state(k), start[masked.case_slice(k)]), k
            assert torch.equal(masked.t_solver.dt[k], dt0[k])
