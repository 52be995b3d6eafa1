"""``TSolver.step_host``: a stream of independent host states, each advanced as if by a freshly
built solver holding it (one CUDA-graph replay per state, the copies overlapped on two copy
streams) -- bitwise equal to building one solver per state."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _states(make, n):
    """n distinct states of the case (the initial one, then every second step)."""
    eq = make(None)
    out = [eq.cells.state.cpu().clone()]
    for _ in range(n - 1):
        eq.t_solver.step(2)
        out.append(eq.cells.state.cpu().clone())
    return out


@pytest.mark.parametrize("case,solver,extra,cfl,steps", [("c2d", "Butcher", "RK4", 0.5, 1),
                                                         ("b3d", "Butcher", "SSP_RK3", 0.5, 2),
                                                         ("c2d", "AB3", "SSP_RK3", None, 4)])
def test_step_host_matches_fresh_solvers(case, solver, extra, cfl, steps):
    from gpu_helpers import make_equation

    def make(state0):
        return make_equation(case, solver, extra, cfl=cfl, state0=state0)[1]

    states = _states(make, 3)
    order = [0, 2, 1, 2, 0]                       # repeats and reordering; 5 > the two slots each way
    inputs = [states[i].pin_memory() for i in order]
    outputs = [torch.full_like(x, float("nan")).pin_memory() for x in inputs]
    eq = make(None)
    eq.t_solver.step(3)                           # leftover gradients / history / dt to be discarded
    eq.t_solver.step_host(inputs, outputs, steps=steps)
    torch.cuda.synchronize()
    for x, y in zip(inputs, outputs):
        ref = make(x.clone())
        ref.t_solver.step(steps)
        torch.cuda.synchronize()
        assert torch.equal(y, ref.cells.state.cpu())
    # the solver holds the last state's result and steps on from it like the fresh one
    ref.t_solver.step(1)
    eq.t_solver.step(1)
    torch.cuda.synchronize()
    assert torch.equal(eq.cells.state, ref.cells.state)
    # a second call reuses the captured graphs; another step count captures new ones
    again = [torch.empty_like(x).pin_memory() for x in inputs[:3]]
    eq.t_solver.step_host(inputs[:3][::-1], again, steps=steps)
    torch.cuda.synchronize()
    for y, z in zip(outputs[:3][::-1], again):
        assert torch.equal(y, z)
    one = [torch.empty_like(inputs[0]).pin_memory()]
    eq.t_solver.step_host(inputs[:1], one, steps=steps + 1)
    torch.cuda.synchronize()
    ref = make(inputs[0].clone())
    ref.t_solver.step(steps + 1)
    torch.cuda.synchronize()
    assert torch.equal(one[0], ref.cells.state.cpu())


def test_step_host_rejects_bad_buffers():
    from gpu_helpers import make_equation
    eq = make_equation("c2d")[1]
    N, C = eq.cells.state.shape
    good = torch.zeros((N, C)).pin_memory()
    with pytest.raises(ValueError):
        eq.t_solver.step_host([good], [])
    with pytest.raises(ValueError):
        eq.t_solver.step_host([torch.zeros((N + 1, C))], [good])
    with pytest.raises(ValueError):
        eq.t_solver.step_host([good], [torch.zeros((N, C), device="cuda")])
    with pytest.raises(ValueError):
        eq.t_solver.step_host([good], [good])
    assert eq.t_solver.step_host([], []) == []
