"""TSolver.solve(): the reference's main loop (t_solvers.py:77-154) -- end time, save cadence in the
reference's Saver format, exact save intervals, NaN check.  Needs a B200."""
import glob
import os

import numpy as np
import pytest
import torch

from gpu_helpers import make_equation

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


def _times(d):
    from fvm_solver_b200 import trajectory_io as tio
    return sorted(float(tio.load_step(p)[0]) for p in glob.glob(os.path.join(d, "t_*.npz")))


def test_solve_end_time_and_saves(tmp_path):
    g, eq, T, cfg = make_equation("c2d", "Butcher", "RK4")
    dt = float(g["dt"])
    sol = eq.t_solver
    sol.cfg.save_t, sol.cfg.save_dir, sol.cfg.plot_t = 1.9 * dt, str(tmp_path), 3 * dt
    sol.n_steps, sol.end_t, sol.print_i = None, 5.5 * dt, 2
    t = sol.solve()
    assert sol.steps_done == 6 and abs(t - 6 * dt) < 1e-6 * dt
    got = _times(tmp_path)
    assert len(got) == 4 and got[0] == 0.0           # t = 0, then the first step past 1.9, 3.8, 5.7 dt
    assert np.allclose(got[1:], [2 * dt, 4 * dt, 6 * dt], rtol=1e-5)
    # the same 6 steps without the loop give the same state
    g2, eq2, _, _ = make_equation("c2d", "Butcher", "RK4")
    eq2.t_solver.step(6)
    assert torch.equal(eq.cells.state, eq2.cells.state)


def test_solve_exact_interval(tmp_path):
    g, eq, T, cfg = make_equation("c2d", "Butcher", "RK4")
    dt = float(g["dt"])
    sol = eq.t_solver
    sol.cfg.save_t, sol.cfg.save_dir, sol.cfg.exact_interval = 2.5 * dt, str(tmp_path), True
    sol.n_steps, sol.end_t, sol.print_i = None, 4.99 * dt, None
    t = sol.solve()
    got = _times(tmp_path)
    assert np.allclose(got, [0.0, 2.5 * dt, 5 * dt], rtol=1e-5)     # steps shortened onto the save times
    assert abs(t - 5 * dt) < 1e-6 * dt
    assert abs(float(sol.dt[0].item()) / dt - 1) < 1e-6               # step size restored afterwards


def test_solve_nan_check():
    g, eq, T, cfg = make_equation("c2d", "Butcher", "RK4")
    st = eq.cells.state.clone()
    st[7, 2] = float("nan")
    eq.cells.state = st
    sol = eq.t_solver
    sol.n_steps, sol.end_t, sol.print_i = 3, None, 1
    with pytest.raises(ValueError, match="Nan"):
        sol.solve()


def test_profile_mode_writes_trace(tmp_path):
    """cfg.profile: the reference's profiling mode -- warm-up, profiled steps, a table of the
    top CUDA entries naming the library's kernels, a Chrome trace file."""
    from gpu_helpers import make_equation
    g, eq, T, cfg = make_equation("c2d", "Butcher", "SSP_RK3")
    path = str(tmp_path / "trace.json")
    table = eq.t_solver.solve_profile(warmup=2, steps=3, trace_path=path)
    assert os.path.getsize(path) > 0
    assert "k_face" in table or "k_cell" in table
    assert eq.t_solver.steps_done == 5
    assert torch.isfinite(eq.cells.state).all()
