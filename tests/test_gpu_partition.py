"""Partitioned (halo-exchange) stepping of one mesh against the single-mesh solver.

The parts run on one GPU through ``LocalComm`` (the ranks of a multi-GPU run, emulated by
sequential launches with device copies for the exchanges).  Every owned cell and facet does the
same arithmetic as in the single-mesh run, so the result is bitwise identical when the mesh has
no characteristic boundary, and equal to FP32 rounding of the cross-part sound-speed mean
otherwise.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run_partitioned(eq, state0, parts_n, steps, cfl):
    from fvm_solver_b200.partition import LocalComm, PartitionedSolver, split_tables
    parts = split_tables(eq.tables.kernel, parts_n)
    ps = PartitionedSolver(parts, LocalComm(parts, "cuda"), eq.phys, eq.t_solver.tab)
    ps.set_state(state0)
    ps.cfl_dt(cfl)
    ps.step(steps)
    out = torch.empty_like(state0)
    ps.gather_state(out)
    torch.cuda.synchronize()
    return out, ps


def _single(eq, steps):
    eq.t_solver.step(steps)
    torch.cuda.synchronize()
    return eq.cells.state.clone()


@pytest.mark.parametrize("parts_n", [2, 3])
def test_partitioned_periodic_box_bitwise(parts_n):
    from fvm_solver_b200 import workloads as W
    case = W.taylor_green(n=10, device="cuda")
    eq = case.equation()
    state0 = eq.cells.state.clone()
    got, ps = _run_partitioned(eq, state0, parts_n, 4, case.cfg.cfl)
    want = _single(eq, 4)
    assert eq.tables.kernel.n_bc == 0
    assert torch.equal(got, want), float((got - want).abs().max())
    assert torch.equal(ps.parts[0].dt, eq.t_solver.dt)


@pytest.mark.parametrize("case_name,parts_n", [("c2d", 2), ("c2d", 4), ("b3d", 3)])
def test_partitioned_golden_meshes(case_name, parts_n):
    from gpu_helpers import make_equation
    g, eq, T, cfg = make_equation(case_name, "Butcher", "RK4", cfl=0.5)
    state0 = eq.cells.state.clone()
    got, ps = _run_partitioned(eq, state0, parts_n, 5, 0.5)
    want = _single(eq, 5)
    kt = eq.tables.kernel
    if kt.n_char == 0:
        assert torch.equal(got, want), float((got - want).abs().max())
    else:
        rel = float((got - want).double().norm() / want.double().norm())
        assert rel < 1e-6, rel
    assert torch.isfinite(got).all()


def test_partitioned_graph_replay_matches_eager():
    from fvm_solver_b200 import workloads as W
    from fvm_solver_b200.partition import LocalComm, PartitionedSolver, split_tables
    case = W.taylor_green(n=8, device="cuda")
    eq = case.equation()
    state0 = eq.cells.state.clone()
    parts = split_tables(eq.tables.kernel, 3)
    outs = []
    for use_graph in (False, True):
        ps = PartitionedSolver(parts, LocalComm(parts, "cuda"), eq.phys, eq.t_solver.tab)
        ps.set_state(state0)
        ps.cfl_dt(case.cfg.cfl)
        if use_graph:
            ps.graph_steps(3)()
        else:
            ps.step(3)
        out = torch.empty_like(state0)
        ps.gather_state(out)
        torch.cuda.synchronize()
        outs.append(out)
    assert torch.equal(outs[0], outs[1])
