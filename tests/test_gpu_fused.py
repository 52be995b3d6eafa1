"""The fused step (one cooperative launch per step, grid barriers between phases) against the
separate launches: bitwise equal states and time steps; the autotuner's choice; barrier status."""
import copy

import pytest
import torch

pytestmark = pytest.mark.gpu


def _pair(make):
    a, b = make(), make()
    b.t_solver.fused = True
    return a, b


@pytest.mark.parametrize("case,solver,extra,cfl", [("c2d", "Butcher", "RK4", 0.5), ("b3d", "Butcher", "SSP_RK3", 0.5),
                                                   ("c2d", "AB3", "SSP_RK3", None)])
def test_fused_step_bitwise(case, solver, extra, cfl):
    from gpu_helpers import make_equation
    a, b = _pair(lambda: make_equation(case, solver, extra, cfl=cfl)[1])
    a.t_solver.step(7)
    b.t_solver.step(5)
    b.t_solver.graph_steps(2)()
    torch.cuda.synchronize()
    assert torch.equal(a.cells.state, b.cells.state)
    assert torch.equal(a.t_solver.dt, b.t_solver.dt)
    assert torch.equal(a.grads, b.grads)
    assert b.t_solver.fused_status() == 0


@pytest.mark.parametrize("case,width", [("c2d", 7), ("b3d", 9), ("b3d", 16)])
def test_fused_step_widened_stencil_bitwise(case, width):
    """Widened gradient stencils (the wide cell body) inside the fused step: bitwise equal too."""
    from gpu_helpers import make_equation
    a, b = _pair(lambda: make_equation(case, "Butcher", "RK4", cfl=0.5, grad_stencil=width)[1])
    assert a.dev.kg > (2 if case == "c2d" else 3) + 2
    a.t_solver.step(4)
    b.t_solver.step(4)
    torch.cuda.synchronize()
    assert torch.equal(a.cells.state, b.cells.state)
    assert torch.equal(a.grads, b.grads)
    assert b.t_solver.fused_status() == 0


def test_fused_adaptive_close():
    from gpu_helpers import make_equation
    a, b = _pair(lambda: make_equation("c2d", "Butcher_adapt", "RK3_SSP4")[1])
    a.t_solver.step(4)
    b.t_solver.step(4)
    torch.cuda.synchronize()
    rel = float((a.cells.state - b.cells.state).double().norm() / a.cells.state.double().norm())
    assert rel < 1e-6
    assert abs(float(a.t_solver.dt[0]) / float(b.t_solver.dt[0]) - 1) < 1e-5


def test_fused_batched_with_case_mask():
    from fvm_solver_b200 import batched as B, workloads as W
    cases = []
    for i, n in enumerate([2100, 3300, 2500]):
        p = W.ensemble_params(i)
        p["n_cells"] = n
        cases.append(W.channel_cylinder(device="cuda", solver_name="AB3", solver_extra="SSP_RK3", cfl=0.3, **p))
    parts = [B.build_case_tables(c) for c in cases]
    a = B.BatchedFVM(parts, cases[0].cfg, device="cuda")
    b = B.BatchedFVM(parts, cases[0].cfg, device="cuda")
    b.t_solver.fused = True
    for x in (a, b):
        x.use_case_mask(True)
        x.active.copy_(torch.tensor([1, 0, 1], dtype=torch.uint8))
        x.t_solver.step(5)
    torch.cuda.synchronize()
    assert torch.equal(a.cells.state, b.cells.state)
    assert torch.equal(a.t_solver.dt, b.t_solver.dt)
    assert b.t_solver.fused_status() == 0


def test_tune_fused_picks_and_restores():
    from fvm_solver_b200 import autotune
    from gpu_helpers import make_equation
    g, eq, T, cfg = make_equation("c2d", "Butcher", "SSP_RK3", cfl=0.5)
    before = eq.cells.state.clone()
    res = autotune.tune_fused(eq, steps=4, reps=2)
    assert set(res["ms_per_step"]) == {"separate", "fused"}
    assert eq.t_solver.fused == res["fused"]
    assert torch.equal(eq.cells.state, before)


def test_grid_barrier_gives_up_and_context_survives():
    """A block that never reaches the barrier: the others' bounded waits end, the status says so,
    and the GPU context keeps working (a fused step runs correctly afterwards)."""
    import ctypes as ct
    from fvm_solver_b200 import _lib
    lib = _lib.load()
    st = ct.c_int32(-1)
    assert lib.fvm_barrier_selftest(8, -1, ct.byref(st)) == 0 and st.value == 0
    st = ct.c_int32(-1)
    assert lib.fvm_barrier_selftest(8, 3, ct.byref(st)) == 0 and st.value == 1
    from gpu_helpers import make_equation
    a, b = _pair(lambda: make_equation("c2d", "Butcher", "RK4", cfl=0.5)[1])
    a.t_solver.step(2)
    b.t_solver.step(2)
    torch.cuda.synchronize()
    assert torch.equal(a.cells.state, b.cells.state) and b.t_solver.fused_status() == 0
