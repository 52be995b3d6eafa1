"""CUDA path vs the reference (golden vectors) and vs the oracle.  Needs a B200.

Tolerances (written per check):
* residuals / limited gradients vs the FP32 reference: rel-L2 <= 1e-5 (FP32 rounding; the
  reference's own FP32-vs-FP64 gap on these cases is ~1e-6 .. 1e-5);
* states after one or ten steps vs the FP32 reference: rel-L2 <= 1e-5 (the per-step parity bar);
* ELL operators vs torch sparse (FP32): rel-L2 <= 1e-6.
The FP64 error of every result is also checked to stay within the reference's own FP32 error x 10.
"""
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2
from gpu_helpers import make_equation, to_np

pytestmark = pytest.mark.gpu

CASES = ["c2d", "b3d"]


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")


# -- ELL operators ----------------------------------------------------------------------------
@pytest.mark.parametrize("K", [1, 2, 5, 16])
@pytest.mark.parametrize("B", [1, 4, 5, 9])
def test_ell_random_vs_torch_sparse(K, B):
    from fvm_solver_b200.sparse import SPMB200
    g = torch.Generator().manual_seed(K * 100 + B)
    M, N = 3001, 2003
    nnz_row = torch.randint(0, K + 1, (M,), generator=g)          # ragged rows incl. empty ones
    rows = torch.repeat_interleave(torch.arange(M), nnz_row)
    cols = torch.randint(0, N, (rows.numel(),), generator=g)
    vals = torch.randn(rows.numel(), generator=g)
    A = torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (M, N)).coalesce()
    op = SPMB200(A, "cuda")
    X = torch.randn(N, B, generator=g).cuda()
    b = torch.randn(M, generator=g).cuda()
    Ad = A.cuda()
    ref = torch.sparse.mm(Ad, X)
    assert rel_l2(to_np(op.spMM(X)), to_np(ref)) < 1e-6
    assert rel_l2(to_np(op.spMM(X, b)), to_np(ref + b[:, None])) < 1e-6
    x = X[:, 0]                                   # strided 1-D view when B > 1
    y = op.spMV(x, b)
    assert y.shape == (M,)
    assert rel_l2(to_np(y), to_np(torch.sparse.mm(Ad, x[:, None])[:, 0] + b)) < 1e-6


def test_ell_empty_and_zero_width():
    from fvm_solver_b200.sparse import SPMB200
    A = torch.sparse_coo_tensor(torch.zeros((2, 0), dtype=torch.long), torch.zeros(0), (7, 5))
    op = SPMB200(A, "cuda")
    x = torch.randn(5, 3, device="cuda")
    assert torch.equal(op.spMM(x), torch.zeros(7, 3, device="cuda"))
    b = torch.arange(7.0, device="cuda")
    assert torch.equal(op.spMV(x[:, 0], b), b)


@pytest.mark.parametrize("case", CASES)
def test_reference_operators_on_device(case):
    """SPMB200 built from the reference-format operators reproduces the oracle ELL products."""
    from fvm_solver_b200.sparse import SPMB200
    from oracle import fvm_oracle as O
    from conftest import golden_setup
    g, spec, T, cfg = golden_setup(case)
    for A in (T.ops.G_mats, T.ops.flux_mat, T.ops.A_face_grad):
        op = SPMB200(A, "cuda")
        v, c = O.ell_from_coo(A)
        X = np.random.default_rng(0).standard_normal((A.shape[1], 4)).astype(np.float32)
        want = O.ell_spmm(v, c, X)
        got = to_np(op.spMM(torch.from_numpy(X).cuda()))
        assert rel_l2(got, want) < 1e-6


# -- residual ------------------------------------------------------------------------------------
@pytest.mark.parametrize("case", CASES)
def test_residual_vs_reference(case):
    g, eq, T, cfg = make_equation(case)
    r1 = eq.forward(torch.from_numpy(g["prim0"]))
    assert rel_l2(to_np(r1), g["res1"]) < 1e-5
    assert rel_l2(to_np(eq.cell_grads), g["grads1"]) < 1e-5
    # second call carries the limited gradients into the boundary correction
    r2 = eq.forward(torch.from_numpy(g["prim2"]))
    assert rel_l2(to_np(r2), g["res2"]) < 1e-5
    assert rel_l2(to_np(eq.cell_grads), g["grads2"]) < 1e-5
    # FP64 error: no worse than 10x the reference's own FP32 error
    e32 = rel_l2(g["res1"], g["res1_f64"])
    eq.reset_gradients()
    r1b = eq.forward(torch.from_numpy(g["prim0"]))
    assert rel_l2(to_np(r1b), g["res1_f64"]) < max(10 * e32, 1e-6)


@pytest.mark.parametrize("case", CASES)
def test_residual_deterministic(case):
    g, eq, T, cfg = make_equation(case)
    p = torch.from_numpy(g["prim0"])
    a = eq.forward(p)
    eq.reset_gradients()
    b = eq.forward(p)
    assert torch.equal(a, b)


# -- integrators ---------------------------------------------------------------------------------
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("extra,key", [("RK4", "rk4_step1"), ("SSP_RK3", "ssprk3_step1")])
def test_butcher_one_step(case, extra, key):
    g, eq, T, cfg = make_equation(case, "Butcher", extra)
    eq.t_solver.step(1)
    st = to_np(eq.cells.state)
    assert rel_l2(st, g[key]) < 1e-5
    assert rel_l2(st, g[key + "_f64"]) < 1e-5


@pytest.mark.parametrize("case", CASES)
def test_ten_steps(case):
    g, eq, T, cfg = make_equation(case, "Butcher", "SSP_RK3")
    eq.t_solver.step(10)
    assert rel_l2(to_np(eq.cells.state), g["ssprk3_step10"]) < 1e-5


@pytest.mark.parametrize("case", ["c2d11k", "b3d9k"])
def test_larger_mesh_vs_reference(case):
    """The larger light fixtures (the 11 307-triangle channel mesh of the channel-cylinder
    benchmark, a 9 066-tet box): first residual and ten SSP-RK3 steps against the reference, FP32
    bar 1e-5; FP64 within 10x the reference's own FP32 error."""
    g, eq, T, cfg = make_equation(case, "Butcher", "SSP_RK3")
    r1 = to_np(eq.forward(torch.from_numpy(g["prim0"])))
    assert rel_l2(r1, g["res1"]) < 1e-5
    assert rel_l2(r1, g["res1_f64"]) < max(10 * rel_l2(g["res1"], g["res1_f64"]), 1e-6)
    eq.reset_gradients()
    eq.t_solver.step(10)
    st = to_np(eq.cells.state)
    assert rel_l2(st, g["ssprk3_step10"]) < 1e-5
    assert rel_l2(st, g["ssprk3_step10_f64"]) < 1e-5


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("name,extra,key", [("Butcher_adapt", "RK3_SSP4", "adapt"), ("RK3_SSP4", "", "rk3ssp4")])
def test_adaptive_step(case, name, extra, key):
    g, eq, T, cfg = make_equation(case, name, extra)
    eq.t_solver.step(1)
    assert rel_l2(to_np(eq.cells.state), g[f"{key}_step1"]) < 1e-5
    dt = float(eq.t_solver.dt.item())
    assert abs(dt / float(g[f"{key}_dt1"]) - 1) < 1e-4


@pytest.mark.parametrize("case", CASES)
def test_ab3_vs_oracle(case):
    from oracle import fvm_oracle as O
    g, eq, T, cfg = make_equation(case, "AB3", "")
    s = O.OracleSolver(O.OracleResidual(T, cfg, np.float32), g["state0"], float(g["dt"]))
    s.ab3_start()
    for _ in range(3):
        s.ab3_step()
    eq.t_solver.step(5)
    assert rel_l2(to_np(eq.cells.state), s.state) < 1e-5


def test_ab3_vs_reference_residual():
    """AB3 (two SSP-RK3 start-up steps, three AB3 steps) against the same scheme driven by the
    reference's own residual (fixture c2dvar): FP32 and FP64 bar 1e-5."""
    g, eq, T, cfg = make_equation("c2dvar", "AB3", "")
    eq.t_solver.step(5)
    st = to_np(eq.cells.state)
    assert rel_l2(st, g["ab3_step5"]) < 1e-5
    assert rel_l2(st, g["ab3_step5_f64"]) < 1e-5


@pytest.mark.parametrize("p", [1, 2, 3, 5])
def test_limiter_variants_vs_reference(p):
    """Limiters p1, p2, p3, p5 (the other cases use p4): residual and limited gradients vs the
    reference, 1e-5."""
    g, eq, T, cfg = make_equation("c2dvar", lim_p=p)
    r1 = eq.forward(torch.from_numpy(g["prim0"]))
    assert rel_l2(to_np(r1), g[f"lim{p}_res1"]) < 1e-5
    assert rel_l2(to_np(eq.cell_grads), g[f"lim{p}_grads1"]) < 1e-5


@pytest.mark.parametrize("name", ["RK3_SSP5", "RK3_SSP6", "RK4_SSP5", "RK4_SSP10"])
def test_tableau_variants_vs_reference(name):
    """One Butcher step with each remaining tableau vs the reference: FP32 and FP64 bar 1e-5."""
    g, eq, T, cfg = make_equation("c2dvar", "Butcher", name)
    eq.t_solver.step(1)
    st = to_np(eq.cells.state)
    assert rel_l2(st, g[f"{name.lower()}_step1"]) < 1e-5
    assert rel_l2(st, g[f"{name.lower()}_step1_f64"]) < 1e-5


def test_periodic_box_vs_unrolled_reference():
    """The benchmark's geometry (periodic Taylor-Green box) against the reference's own geometry:
    the central tile of the box unrolled 3 x 3 x 3 and run through the reference's FVMMesh3D /
    FVMEquation.forward (fixture ptile).  Residual, limited gradients and one RK4 step: 1e-5, the
    per-step parity bar; the RK4 step also against the FP64 reference."""
    g, eq, T, cfg = make_equation("ptile", "Butcher", "RK4")
    r1 = eq.forward(torch.from_numpy(g["prim0"]))
    assert rel_l2(to_np(r1), g["res1"]) < 1e-5
    assert rel_l2(to_np(eq.cell_grads), g["grads1"]) < 1e-5
    eq.reset_gradients()
    eq.t_solver.step(1)
    st = to_np(eq.cells.state)
    assert rel_l2(st, g["rk4_step1"]) < 1e-5
    assert rel_l2(st, g["rk4_step1_f64"]) < 1e-5


@pytest.mark.parametrize("case", CASES)
def test_cfl_and_conservation(case):
    from oracle import fvm_oracle as O
    g, eq, T, cfg = make_equation(case, "Butcher", "SSP_RK3", cfl=0.5)
    want = O.cfl_dt(g["state0"], int(g["dim"]), cfg.C_v, cfg.gamma, T.kernel.inv_h.numpy(), 0.5)
    got = float(eq.t_solver.dt.item())
    assert abs(got / want - 1) < 1e-6
    tot = to_np(eq.conservation())
    vol = T.kernel.volumes.numpy()
    want_tot = (vol[:, None] * g["state0"].astype(np.float64)).sum(0)
    assert np.allclose(tot, want_tot, rtol=1e-12, atol=1e-9)
    # CFL after a step is computed in the step's last stage kernel
    eq.t_solver.step(1)
    want = O.cfl_dt(to_np(eq.cells.state), int(g["dim"]), cfg.C_v, cfg.gamma, T.kernel.inv_h.numpy(), 0.5)
    assert abs(float(eq.t_solver.dt.item()) / want - 1) < 1e-6


@pytest.mark.parametrize("case", CASES)
def test_graph_replay_matches_eager(case):
    g, eq, T, cfg = make_equation(case, "Butcher", "RK4", cfl=0.5)
    g2, eq2, _, _ = make_equation(case, "Butcher", "RK4", cfl=0.5)
    eq.t_solver.step(4)
    replay = eq2.t_solver.graph_steps(2)
    replay()
    replay()
    assert torch.equal(eq.cells.state, eq2.cells.state)
    assert torch.equal(eq.t_solver.dt, eq2.t_solver.dt)


def test_periodic_box_vs_oracle():
    """Periodic tetrahedral box (no reference counterpart): CUDA path vs oracle, residual and step."""
    from fvm_solver_b200 import config as cf, equation as E, fvm_mesh as fm, meshgen as mg, tables as tb
    from oracle import fvm_oracle as O
    spec = mg.periodic_box(8, seed=5)
    cfg = cf.TaylorGreenConfig(device="cuda")
    tabs = tb.FVMTables(fm.mesh_from_spec(spec), cfg, 5, {})
    rng = np.random.default_rng(1)
    N = spec.n_cells
    prim = np.zeros((N, 5), np.float32)
    prim[:, :3] = rng.standard_normal((N, 3)) * 0.5
    prim[:, 3] = 1 + 0.05 * rng.standard_normal(N)
    prim[:, 4] = 100 + rng.standard_normal(N)
    phy = E.FluidConstitution3D(cfg)
    eq = E.FVMEquation(cfg, phy, spec, 5, {}, us_init=torch.from_numpy(O.prim_to_state(prim, 3, cfg.C_v)))
    orc = O.OracleResidual(tabs, cfg, np.float32)
    want, wg = orc.forward(prim)
    got = eq.forward(torch.from_numpy(prim))
    assert rel_l2(to_np(got), want) < 1e-5
    assert rel_l2(to_np(eq.cell_grads), wg) < 1e-5


def test_free_stream_preservation_periodic():
    """Uniform flow on a periodic mesh: every facet flux is identical, so dU/dt ~ 0 (size-independent)."""
    from fvm_solver_b200 import config as cf, equation as E, meshgen as mg
    spec = mg.periodic_box(24, seed=2)
    cfg = cf.TaylorGreenConfig(device="cuda")
    phy = E.FluidConstitution3D(cfg)
    N = spec.n_cells
    prim = torch.zeros(N, 5)
    prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 3], prim[:, 4] = 0.7, -0.3, 0.2, 1.0, 100.0
    V, rho, T = prim[:, :3], prim[:, 3:4], prim[:, 4:]
    m, r, Q = phy.primatives_to_state(V, rho, T)
    eq = E.FVMEquation(cfg, phy, spec, 5, {}, us_init=torch.cat([m, r, Q], 1))
    d = eq.forward(prim)
    scale = float(eq.tables.kernel.f_vals.abs().max()) * 250.0   # |flux| ~ rho E u |S|
    assert float(d.abs().max()) < 1e-4 * scale


def test_block_size_invariance_and_autotune():
    """Residuals do not depend on the launch configuration; the autotuner installs a valid one."""
    from fvm_solver_b200 import autotune
    g, eq, T, cfg = make_equation("b3d")
    p = torch.from_numpy(g["prim0"]).cuda()
    outs = []
    try:
        for bs in (64, 128, 256, 512):
            for pf in (0, 1, 3, "staged"):
                for k in ("cell", "face", "div_stage"):
                    autotune.set_block_size(k, bs)
                    autotune.set_prefetch(k, 0 if pf == "staged" else pf)
                autotune.set_variant("face", 1 if pf == "staged" else 0)
                eq.reset_gradients()
                outs.append(eq.forward(p))
        assert all(torch.equal(outs[0], o) for o in outs)
        best = autotune.autotune(eq, reps=2, use_cache=False)
        assert set(best) == {"cell", "face", "div_stage"}
        assert all(v["threads"] in autotune.CANDIDATES for v in best.values())
        assert all(v["prefetch"] in autotune.PREFETCH for v in best.values())
        assert best["face"]["variant"] in ("registers", "staged")
        eq.reset_gradients()
        assert torch.equal(eq.forward(p), outs[0])
    finally:
        autotune.reset()
    with pytest.raises(RuntimeError):
        autotune.set_block_size("cell", 48)
    with pytest.raises(RuntimeError):
        autotune.set_prefetch("face", -2)


@pytest.mark.parametrize("name,extra", [("Butcher", "RK4"), ("Butcher_adapt", "RK3_SSP4"), ("AB3", "")])
def test_checkpoint_restart_bitwise(tmp_path, name, extra):
    """Stop after 3 steps, checkpoint, restart in a fresh solver: identical to 6 uninterrupted steps."""
    g, eq, T, cfg = make_equation("c2d", name, extra, cfl=0.5 if name != "Butcher_adapt" else None)
    eq.t_solver.step(6)
    g2, eq2, _, _ = make_equation("c2d", name, extra, cfl=0.5 if name != "Butcher_adapt" else None)
    eq2.t_solver.step(3)
    path = str(tmp_path / "ckpt.pt")
    eq2.t_solver.save_checkpoint(path)
    g3, eq3, _, _ = make_equation("c2d", name, extra, cfl=0.5 if name != "Butcher_adapt" else None)
    eq3.t_solver.load_checkpoint(path)
    eq3.t_solver.step(3)
    assert torch.equal(eq3.cells.state, eq.cells.state)
    assert torch.equal(eq3.t_solver.dt, eq.t_solver.dt)


def test_saver_boundary_values_vs_oracle(tmp_path):
    """Saved boundary-facet values = mean of the facet's two sides, as the oracle computes them."""
    from fvm_solver_b200 import trajectory_io as tio
    from oracle import fvm_oracle as O
    g, eq, T, cfg = make_equation("c2d")
    prims = torch.from_numpy(g["prim0"]).cuda()
    got = tio.boundary_face_values(eq, prims).cpu().numpy()
    _, _, faces = O.OracleResidual(T, cfg, np.float32).forward(g["prim0"], return_faces=True)
    want = faces[T.bc_locations.numpy().astype(np.int64)].mean(axis=1)
    assert rel_l2(got, want) < 1e-5
    saver = tio.TrajectorySaver(eq, str(tmp_path))
    path = saver.save(0.5)
    t, cell, bc = tio.load_step(path)
    assert bc.shape == (T.n_bc, 4) and os.path.exists(str(tmp_path / "mesh_props.npz"))


@pytest.mark.parametrize("case", CASES)
def test_residual_from_state_vs_reference(case):
    """fvm_residual_state (conserved state in, one conversion kernel, then the residual) against the
    reference's residual of the same state's primitives: 1e-5 (the conversion rounds like the
    stage kernels' rather than like the reference's torch ops)."""
    import ctypes as ct
    from fvm_solver_b200 import _lib
    g, eq, T, cfg = make_equation(case)
    st = torch.from_numpy(g["state0"]).cuda().contiguous()
    out = torch.empty_like(st)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    grads = torch.zeros_like(eq.grads)
    _lib.check(eq.lib.fvm_residual_state(ct.byref(eq.dev.struct), ct.byref(eq.phys), st.data_ptr(), grads.data_ptr(),
                                         flag.data_ptr(), out.data_ptr(), ct.byref(eq.work.struct),
                                         _lib.stream_ptr()), "fvm_residual_state")
    assert rel_l2(to_np(out), g["res1"]) < 1e-5
    assert int(flag.item()) == 1


@pytest.mark.parametrize("case", CASES)
def test_facet_state_vs_oracle(case):
    """FVMEquation.facet_state: both sides of every facet (Vs/rho/T_facet, the reference's
    U_face_all, facet_process.py:349-359) and phi against the oracle's facet values, 1e-5."""
    from oracle import fvm_oracle as O
    g, eq, T, cfg = make_equation(case)
    fs = eq.facet_state(torch.from_numpy(g["prim0"]))
    _, _, faces = O.OracleResidual(T, cfg, np.float32).forward(g["prim0"], return_faces=True)
    dim = int(g["dim"])
    got = torch.cat([fs.Vs_facet, fs.rho_facet, fs.T_facet], -1)
    assert rel_l2(to_np(got), faces) < 1e-5
    phi = (faces[:, :, :dim] * T.normals.numpy()[:, None, :]).sum(-1)
    assert rel_l2(to_np(fs.phi), phi) < 1e-5
    assert rel_l2(to_np(fs.cell_grads), g["grads1"]) < 1e-5
    assert eq.cell_grads is None              # the equation's carried gradients are untouched


@pytest.mark.parametrize("case", ["c2d", "b3d", "ptile"])
@pytest.mark.parametrize("width", [9, 16])
def test_widened_stencil_vs_oracle(case, width):
    """Widened gradient stencils (up to 16 slots; no reference counterpart, the reference's width is
    dim + 2): the generic-width cell kernel against the oracle on the same tables -- residual and
    limited gradients 1e-5, one RK4 step 1e-5."""
    from oracle import fvm_oracle as O
    g, eq, T, cfg = make_equation(case, "Butcher", "RK4", grad_stencil=width)
    assert eq.dev.kg > int(g["dim"]) + 2
    orc = O.OracleResidual(eq.tables, cfg, np.float32)
    want, wg = orc.forward(g["prim0"])
    got = eq.forward(torch.from_numpy(g["prim0"]))
    assert rel_l2(to_np(got), want) < 1e-5
    assert rel_l2(to_np(eq.cell_grads), wg) < 1e-5
    eq.reset_gradients()
    eq.t_solver.step(1)
    s = O.OracleSolver(orc, g["state0"], float(g["dt"]))
    s.butcher_step("RK4")
    assert rel_l2(to_np(eq.cells.state), s.state) < 1e-5


@pytest.mark.parametrize("case", ["c2d", "b3d", "ptile"])
def test_owner_computes_residual_bitwise(case):
    """The owner-computes divergence (each cell evaluates its own facets, no flux array) gives the
    bits of facet kernel + divergence kernel, from primitives and from a conserved state."""
    import ctypes as ct
    from fvm_solver_b200 import _lib, autotune
    g, eq, T, cfg = make_equation(case)
    p = torch.from_numpy(g["prim0"]).cuda()
    U = torch.from_numpy(g["state0"]).cuda().contiguous()
    outs = {}
    try:
        for v in (0, 1):
            autotune.set_variant("div_stage", v)
            for bs in (64, 256):
                autotune.set_block_size("face", bs)
                eq.reset_gradients()
                r = eq.forward(p).clone()
                rs = torch.empty_like(U)
                flag = torch.zeros(1, dtype=torch.int32, device="cuda")
                grads = torch.zeros_like(eq.grads)
                _lib.check(eq.lib.fvm_residual_state(ct.byref(eq.dev.struct), ct.byref(eq.phys), U.data_ptr(),
                                                     grads.data_ptr(), flag.data_ptr(), rs.data_ptr(),
                                                     ct.byref(eq.work.struct), _lib.stream_ptr()),
                           "fvm_residual_state")
                outs[(v, bs)] = (r, rs)
    finally:
        autotune.reset()
    ref = outs[(0, 256)]
    for k, (r, rs) in outs.items():
        assert torch.equal(r, ref[0]), k
        assert torch.equal(rs, ref[1]), k
    with pytest.raises(RuntimeError):
        autotune.set_variant("div_stage", 2)


@pytest.mark.parametrize("case,solver,extra", [("c2d", "Butcher", "SSP_RK3"), ("b3d", "Butcher", "RK4"),
                                               ("c2d", "AB3", "")])
def test_launch_overlap_bitwise(case, solver, extra):
    """Programmatic dependent launches (each stage kernel launched while its predecessor drains,
    waiting on the device) change nothing: eager steps and graph-replayed steps with the overlap
    on equal those with it off, bit for bit."""
    from fvm_solver_b200 import autotune
    outs = []
    try:
        for on in (False, True):
            autotune.set_launch_overlap(on)
            g, eq, T, cfg = make_equation(case, solver, extra, cfl=0.5 if solver != "AB3" else None)
            eq.t_solver.step(3)
            eq.t_solver.graph_steps(3)()
            torch.cuda.synchronize()
            outs.append((eq.cells.state.clone(), eq.grads.clone(), eq.t_solver.dt.clone()))
    finally:
        autotune.set_launch_overlap(True)
    for a, b in zip(*outs):
        assert torch.equal(a, b)
