"""Generate the golden fixtures by running the reference implementation (CPU path).

Run where the reference sources are, with ``FVM_REFERENCE_PATH`` naming the checkout (the
directory that holds ``time_fvm/``)::

    FVM_REFERENCE_PATH=<checkout> python tests/golden/make_golden.py [--case NAME ...]
    # writes tests/golden/fvm_golden_<case>.npz; NAME in c2d, b3d (default), c2d11k, b3d9k,
    # c2dvar, ptile

For each case (2D channel-cylinder mesh, 3D box mesh; ``--case c2d11k`` / ``--case b3d9k`` add
the 2D mesh at the channel-cylinder benchmark's size and a 9 066-tet box, stored light: the
state, the first residual and the state after ten SSP-RK3 steps, FP32 and FP64) the script

* builds the mesh with this package's generator and the reference's ``FVMMesh2D/3D``;
* stores the reference's packed ELL operators (``csr_to_ell`` of G_mats, flux_mat,
  A_face_grad, A_bc, A_corr) and offset vectors -> pins the host table build bit-for-bit;
* evaluates ``FVMEquation.forward`` twice (first call without, second with the carried
  ``cell_grads``) and stores residuals and limited gradients;
* takes one step with ``Butcher`` (RK4, and the three-stage SSP-RK3 tableau injected into a
  ``Butcher`` instance), one ``ButcherAdapt`` RK3_SSP4 step (with the updated ``dt``), one step of
  the hand-unrolled ``RK3_SSP4`` class, and ten SSP-RK3 steps;
* repeats the residual and step evaluations in FP64 in a subprocess under a dtype shim
  (keys suffixed ``_f64``).

Two further fixtures pin what the four cases above leave to the oracle:

* ``--case c2dvar`` (the c2d mesh and state): the first residual with the limiters p = 1, 2, 3, 5
  (``limiter.py:29-77``; the cases above use the default p = 4), one ``Butcher`` step with each of
  the tableaus RK3_SSP5, RK3_SSP6, RK4_SSP5 and RK4_SSP10 (``integrators.py:240-296``), and
  Adams-Bashforth 3 driven by the reference's own residual: two SSP-RK3 start-up steps through
  ``Butcher._step`` (the three-stage tableau injected) whose first-stage residuals f(U_n) are
  recorded as they are computed, then three steps U += dt (23 f_n - 16 f_{n-1} + 5 f_{n-2}) / 12
  with f from ``TSolver._forward_state`` (``t_solvers.py:212-215``).  The reference's own
  ``Adams3PC`` cannot run (``integrators.py:111``), so the multistep combination is restated here;
  every residual in it is the reference's.
* ``--case ptile`` (a periodic Taylor-Green box, the geometry of the 3D benchmark): the reference
  has no periodic meshes, so a 6^3-point ``meshgen.periodic_box`` is unrolled into 3 x 3 x 3 tiles
  (explicit vertex copies at lattice shifts, a plain non-periodic tetrahedral mesh of ~40k cells,
  outer faces characteristic inlets) and run through the reference's ``FVMMesh3D`` +
  ``FVMEquation.forward`` with the periodic state repeated in every tile.  The central tile's cells
  come first and keep the periodic numbering; their residual needs cells two neighbours away and one
  RK4 step eight, all inside the tile ring, so the central tile's residual, limited gradients and
  RK4 step are the periodic mesh's answer computed by the reference on its own geometry.  Stored:
  the periodic mesh (vertices, cells, facets, lattice shifts), its state and those central-tile
  results (the outer tiles differ by ~0.2 rel-L2 in their residual, so the ring is what shields
  the centre).
"""
from __future__ import annotations

import argparse
import itertools
import os
import subprocess
import sys
import tempfile

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from refimport import import_reference  # noqa: E402

SSP_RK3 = (torch.tensor([[0.0, 0, 0], [1.0, 0, 0], [0.25, 0.25, 0]]),
           torch.tensor([1 / 6, 1 / 6, 2 / 3]))


def case_spec(case):
    from fvm_solver_b200 import meshgen as mg
    if case == "c2d":
        return mg.channel_cylinder(h=0.05, seed=3), 2
    if case == "c2d11k":                    # the channel-cylinder benchmark's size (h = 0.02)
        return mg.channel_cylinder(h=0.02, seed=3), 2
    if case == "b3d":
        return mg.box3d(6, seed=4), 3
    if case == "b3d9k":
        return mg.box3d(11, seed=4), 3
    raise ValueError(case)


# Cases stored without the ELL operators and with fewer results, to keep the fixture small.
LIGHT = {"c2d11k": (("state0", "res1", "ssprk3_step10"), ("res1", "ssprk3_step10")),
         "b3d9k": (("state0", "res1", "ssprk3_step10"), ("res1", "ssprk3_step10"))}


def initial_prims(spec, dim, seed=11):
    """Smooth + random perturbations so that limiter, gradients and BCs are all active."""
    g = torch.Generator().manual_seed(seed)
    N = spec.n_cells
    x = spec.vertices[spec.cells.long()].mean(1)
    prim = torch.zeros(N, dim + 2)
    prim[:, 0] = 3.0 + 0.5 * torch.sin(3 * x[:, 0]) + 0.2 * torch.randn(N, generator=g)
    prim[:, 1] = 0.4 * torch.cos(2 * x[:, 1]) + 0.2 * torch.randn(N, generator=g)
    if dim == 3:
        prim[:, 2] = 0.3 * torch.sin(2 * x[:, 2]) + 0.2 * torch.randn(N, generator=g)
    prim[:, dim] = 1.0 + 0.1 * torch.sin(2 * x[:, 0] + x[:, 1]) + 0.02 * torch.randn(N, generator=g)
    prim[:, dim + 1] = 100.0 + 5 * torch.cos(x[:, 0]) + 1.0 * torch.randn(N, generator=g)
    return prim


def ref_config(R, dim, solver_name="Butcher", solver_extra="RK4", dt=1e-4):
    cfg = R["config_fvm"].ConfigEllipse()
    cfg.device = "cpu"
    cfg.compile = False
    cfg.plot = False
    cfg.save_dir = tempfile.mkdtemp(prefix="fvm_golden_")
    cfg.solver_name, cfg.solver_extra, cfg.dt = solver_name, solver_extra, dt
    if dim == 3:
        cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
        cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
    return cfg


def build_equation(R, spec, dim, cfg, us, dtype):
    RM, st = R["fvm_mesh"], R["mesh_store"]
    E, Facet = st.FacetBCTypes, st.Facet
    cls = RM.FVMMesh2D if dim == 2 else RM.FVMMesh3D
    mesh = cls(spec.vertices.to(dtype), spec.cells, spec.facets, spec.bc_facet_mask, device="cpu")
    bc = {}
    for i, tg in enumerate(spec.bc_tags):
        if tg == "NavierWall":
            bc[i] = Facet([E.Dirich] * dim + [E.Neuman] * 2, [0.0] * dim + [None, None],
                          [None] * dim + [0, 0], tag=tg)
        elif tg in ("Left", "Farfield"):
            bc[i] = Facet([E.Inlet] * (dim + 2), tag=tg)
        else:
            bc[i] = Facet([E.Farfield] * (dim + 2), tag=tg)
    FE = R["fvm_equation"]
    phy = FE.FluidConstitution2D(cfg, 2) if dim == 2 else FE.FluidConstitution3D(cfg, 3)
    return FE.FVMEquation(cfg, phy, mesh, dim + 2, bc, us_init=us.to(dtype)), phy


def run_reference(case, prim0, dt, fp64):
    R = import_reference(fp64=fp64)
    dtype = torch.float64 if fp64 else torch.float32
    spec, dim = case_spec(case)
    out = {}
    prim0 = prim0.to(dtype)
    cfg = ref_config(R, dim, dt=dt)
    FE = R["fvm_equation"]
    phy = FE.FluidConstitution2D(cfg, 2) if dim == 2 else FE.FluidConstitution3D(cfg, 3)
    V, rho, T = prim0[:, :dim], prim0[:, dim:dim + 1], prim0[:, dim + 1:]
    m, r, Q = phy.primatives_to_state(V, rho, T)
    U0 = torch.cat([m, r, Q], -1)
    out["state0"] = U0
    eq, _ = build_equation(R, spec, dim, cfg, U0, dtype)

    if not fp64 and case not in LIGHT:
        ek = R["ell_kernel"]
        M, BS = eq.E_props.mesh, eq.E_props.boundary_setter
        for name, spm in [("G", M.G_mats), ("flux", eq.flux_mat), ("Afg", M.A_face_grad),
                          ("Abc", BS.A_bc), ("Acorr", BS.A_corr)]:
            v, c = ek.csr_to_ell(spm.A)
            out[f"ell_{name}_vals"], out[f"ell_{name}_cols"] = v, c.long()
        out["b_face_grad"] = M.b_face_grad
        bmask = (eq.E_props.dirich_mask if hasattr(eq.E_props, "dirich_mask") else None)
        out["b_bc"] = BS.b_bc

    with torch.inference_mode():
        eq.E_props.cell_grads = None
        out["res1"] = eq.forward(prim0.clone())
        out["grads1"] = eq.E_props.cell_grads.clone()
        prim2 = prim0 * 1.001
        out["prim2"] = prim2
        out["res2"] = eq.forward(prim2.clone())
        out["grads2"] = eq.E_props.cell_grads.clone()

        ts = eq.t_solver
        # RK4, one step
        eq.E_props.cell_grads = None
        eq.cells.state = U0.clone()
        ts.dt = torch.tensor(dt, dtype=dtype)
        ts._solve_step(torch.tensor(0.0))
        out["rk4_step1"] = eq.cells.state.clone()
        out["rk4_grads1"] = eq.E_props.cell_grads.clone()
        # SSP-RK3 (three-stage tableau injected into Butcher)
        ts.A, ts.b = SSP_RK3[0].to(dtype), SSP_RK3[1].to(dtype).reshape(-1, 1, 1)
        ts.stages = 3
        eq.E_props.cell_grads = None
        eq.cells.state = U0.clone()
        ts._solve_step(torch.tensor(0.0))
        out["ssprk3_step1"] = eq.cells.state.clone()
        for _ in range(9):
            ts._solve_step(torch.tensor(0.0))
        out["ssprk3_step10"] = eq.cells.state.clone()

    # ButcherAdapt RK3_SSP4 and the RK3_SSP4 class
    for sname, sextra, key in ([] if case in LIGHT else
                               [("Butcher_adapt", "RK3_SSP4", "adapt"), ("RK3_SSP4", "", "rk3ssp4")]):
        cfg2 = ref_config(R, dim, sname, sextra, dt)
        eq2, _ = build_equation(R, spec, dim, cfg2, U0, dtype)
        with torch.inference_mode():
            eq2.E_props.cell_grads = None
            eq2.t_solver._solve_step(torch.tensor(0.0))
        out[f"{key}_step1"] = eq2.cells.state.clone()
        out[f"{key}_dt1"] = eq2.t_solver.dt.clone()
    return {k: v.detach().cpu().numpy() for k, v in out.items()}


VARIANT_LIMITERS = (1, 2, 3, 5)
VARIANT_TABLEAUS = ("RK3_SSP5", "RK3_SSP6", "RK4_SSP5", "RK4_SSP10")
AB3_COEF = (23 / 12, -16 / 12, 5 / 12)


def run_variants(prim0, dt, fp64):
    """The ``c2dvar`` results on the c2d mesh: other limiters, other tableaus, AB3."""
    R = import_reference(fp64=fp64)
    dtype = torch.float64 if fp64 else torch.float32
    spec, dim = case_spec("c2d")
    prim0 = prim0.to(dtype)
    out = {}
    for p in VARIANT_LIMITERS:
        cfg = ref_config(R, dim, dt=dt)
        cfg.lim_p = p
        FE = R["fvm_equation"]
        phy = FE.FluidConstitution2D(cfg, 2)
        m, r, Q = phy.primatives_to_state(prim0[:, :dim], prim0[:, dim:dim + 1], prim0[:, dim + 1:])
        eq, _ = build_equation(R, spec, dim, cfg, torch.cat([m, r, Q], -1), dtype)
        with torch.inference_mode():
            eq.E_props.cell_grads = None
            out[f"lim{p}_res1"] = eq.forward(prim0.clone())
            out[f"lim{p}_grads1"] = eq.E_props.cell_grads.clone()
    for name in VARIANT_TABLEAUS:
        cfg = ref_config(R, dim, "Butcher", name, dt)
        FE = R["fvm_equation"]
        phy = FE.FluidConstitution2D(cfg, 2)
        m, r, Q = phy.primatives_to_state(prim0[:, :dim], prim0[:, dim:dim + 1], prim0[:, dim + 1:])
        U0 = torch.cat([m, r, Q], -1)
        eq, _ = build_equation(R, spec, dim, cfg, U0, dtype)
        with torch.inference_mode():
            eq.E_props.cell_grads = None
            eq.t_solver.dt = torch.tensor(dt, dtype=dtype)
            eq.t_solver._solve_step(torch.tensor(0.0))
        out[f"{name.lower()}_step1"] = eq.cells.state.clone()
    # Adams-Bashforth 3 on the reference's residual
    cfg = ref_config(R, dim, "Butcher", "RK4", dt)
    FE = R["fvm_equation"]
    phy = FE.FluidConstitution2D(cfg, 2)
    m, r, Q = phy.primatives_to_state(prim0[:, :dim], prim0[:, dim:dim + 1], prim0[:, dim + 1:])
    U0 = torch.cat([m, r, Q], -1)
    eq, _ = build_equation(R, spec, dim, cfg, U0, dtype)
    ts = eq.t_solver
    ts.A, ts.b = SSP_RK3[0].to(dtype), SSP_RK3[1].to(dtype).reshape(-1, 1, 1)
    ts.stages = 3
    ts.dt = torch.tensor(dt, dtype=dtype)
    forward_state = ts._forward_state
    seen = []

    def recording(U):
        f = forward_state(U)
        seen.append(f)
        return f

    hist = []                                 # dt * f(U_n), newest last
    with torch.inference_mode():
        eq.E_props.cell_grads = None
        ts._forward_state = recording
        for _ in range(2):                    # SSP-RK3 start-up; its first stage is f(U_n)
            seen.clear()
            ts._solve_step(torch.tensor(0.0))
            hist.append(ts.dt * seen[0])
        ts._forward_state = forward_state
        for _ in range(3):
            U = eq.cells.state
            hist.append(ts.dt * forward_state(U))
            inc = AB3_COEF[0] * hist[-1] + AB3_COEF[1] * hist[-2] + AB3_COEF[2] * hist[-3]
            eq.cells.update_cells(U + inc)
    out["ab3_step5"] = eq.cells.state.clone()
    return {k: v.detach().cpu().numpy() for k, v in out.items()}


PTILE_N, PTILE_SEED, PTILE_NOISE_SEED = 6, 7, 11


def tile_periodic(spec, reps: int = 3):
    """Unroll a periodic ``MeshSpec`` into reps^3 copies of the box (reps odd): vertex copies at the
    lattice shifts each tile needs, cells of the central tile first (periodic numbering), then the
    other tiles; facets interior first, then boundary.  Returns (vertices f32, cells, facets,
    bc mask, number of tiles)."""
    P = spec.vertices.numpy().astype(np.float64)
    L = float(spec.period[0])
    cells = spec.cells.numpy().astype(np.int64)
    csh = spec.cell_shifts.numpy().astype(np.int64)
    h = reps // 2
    tiles = [np.zeros(3, np.int64)] + [np.array(t) for t in itertools.product(range(-h, h + 1), repeat=3) if any(t)]
    base = 2 * h + 3                         # shifts of a tile vertex lie in [-(h + 1), h + 1]
    keys = np.concatenate([cells * base ** 3 + ((csh + t) + h + 1) @ np.array([base * base, base, 1])
                           for t in tiles])
    uniq, inv = np.unique(keys.reshape(-1), return_inverse=True)
    tcells = inv.reshape(-1, 4)
    vid, rem = uniq // base ** 3, uniq % base ** 3
    shift = np.stack([rem // (base * base), (rem // base) % base, rem % base], 1) - (h + 1)
    verts = (P[vid] + shift * L).astype(np.float32)
    pats = [(0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 3, 2)]
    loc = np.sort(np.stack([tcells[:, list(p)] for p in pats], 1).reshape(-1, 3), axis=1)
    uq, cnt = np.unique(loc, axis=0, return_counts=True)
    assert cnt.max() <= 2, "non-manifold facet"
    facets = np.concatenate([uq[cnt == 2], uq[cnt == 1]])
    mask = np.concatenate([np.zeros(int((cnt == 2).sum()), bool), np.ones(int((cnt == 1).sum()), bool)])
    return verts, tcells.astype(np.int32), facets.astype(np.int64), mask, len(tiles)


def ptile_inputs():
    """The periodic box, its perturbed Taylor-Green state and the CFL 0.5 time step."""
    from fvm_solver_b200 import fvm_mesh as fm, meshgen as mg, tables as tb, workloads as W
    from oracle.fvm_oracle import cfl_dt, prim_to_state, state_to_prim
    case = W.taylor_green(n=PTILE_N, seed=PTILE_SEED, device="cpu")
    spec, cfg = case.spec, case.cfg
    N = spec.n_cells
    rng = np.random.default_rng(PTILE_NOISE_SEED)     # perturbations that switch the limiter on
    prim = state_to_prim(case.state0.numpy().astype(np.float64), 3, cfg.C_v)
    prim[:, :3] += 0.1 * cfg.v0 * rng.standard_normal((N, 3))
    prim[:, 3] *= 1 + 0.02 * rng.standard_normal(N)
    prim[:, 4] *= 1 + 0.01 * rng.standard_normal(N)
    prim = prim.astype(np.float32)
    T = tb.FVMTables(fm.mesh_from_spec(spec), cfg, 5, {})
    U0 = prim_to_state(prim.astype(np.float64), 3, cfg.C_v).astype(np.float32)
    dt = float(cfl_dt(U0.astype(np.float64), 3, cfg.C_v, cfg.gamma, T.kernel.inv_h.numpy(), 0.5))
    return spec, cfg, prim, dt


def run_ptile(tiled, prim0, dt, fp64):
    """Residual, limited gradients and one RK4 step of the unrolled periodic box (reference)."""
    from fvm_solver_b200 import config as cf
    R = import_reference(fp64=fp64)
    dtype = torch.float64 if fp64 else torch.float32
    verts, tcells, facets, mask, n_tiles = tiled
    tg = cf.TaylorGreenConfig(device="cpu")
    cfg = ref_config(R, 3, "Butcher", "RK4", dt)
    for k in ("T_0", "viscosity", "visc_bulk", "thermal_cond", "S_const", "gamma", "C_v", "v_factor",
              "lim_p", "lim_K"):
        setattr(cfg, k, getattr(tg, k))
    cfg.inlet_cfg.v_inf = (0.0, 0.0, 0.0)
    cfg.exit_cfg.v_inf = (0.0, 0.0, 0.0)
    st = R["mesh_store"]
    E = st.FacetBCTypes
    mesh = R["fvm_mesh"].FVMMesh3D(torch.from_numpy(verts).to(dtype), torch.from_numpy(tcells),
                                   torch.from_numpy(facets), torch.from_numpy(mask), device="cpu")
    bc = {i: st.Facet([E.Inlet] * 5, tag="Farfield") for i in range(int(mask.sum()))}
    FE = R["fvm_equation"]
    phy = FE.FluidConstitution3D(cfg, 3)
    prim = torch.from_numpy(np.tile(prim0, (n_tiles, 1))).to(dtype)
    m, r, Q = phy.primatives_to_state(prim[:, :3], prim[:, 3:4], prim[:, 4:])
    U0 = torch.cat([m, r, Q], -1)
    eq = FE.FVMEquation(cfg, phy, mesh, 5, bc, us_init=U0)
    N = prim0.shape[0]
    out = {}
    with torch.inference_mode():
        eq.E_props.cell_grads = None
        out["res1"] = eq.forward(prim.clone())[:N]
        out["grads1"] = eq.E_props.cell_grads[:N].clone()
        eq.E_props.cell_grads = None
        eq.cells.state = U0.clone()
        eq.t_solver.dt = torch.tensor(dt, dtype=dtype)
        eq.t_solver._solve_step(torch.tensor(0.0))
        out["rk4_step1"] = eq.cells.state[:N].clone()
    return {k: v.detach().cpu().numpy() for k, v in out.items()}


def make_variants():
    g = dict(np.load(os.path.join(HERE, "fvm_golden_c2d.npz")))
    prim0, dt = torch.from_numpy(g["prim0"]), float(g["dt"])
    res32 = run_variants(prim0, dt, fp64=False)
    res64 = _fp64_subprocess("c2dvar", dict(prim0=g["prim0"], dt=dt))
    out = {k: g[k] for k in ("prim0", "dt", "state0", "vertices", "cells", "facets", "bc_facet_mask", "bc_tags",
                             "dim")}
    out.update(res32)
    out.update({k + "_f64": v for k, v in res64.items()})
    return out


def make_ptile():
    spec, cfg, prim, dt = ptile_inputs()
    tiled = tile_periodic(spec, 3)
    res32 = run_ptile(tiled, prim, dt, fp64=False)
    verts, tcells, facets, mask, n_tiles = tiled
    res64 = _fp64_subprocess("ptile", dict(prim0=prim, dt=dt, verts=verts, tcells=tcells, facets=facets,
                                           mask=mask, n_tiles=n_tiles))
    from oracle.fvm_oracle import prim_to_state
    out = dict(prim0=prim, dt=np.float64(dt), state0=prim_to_state(prim.astype(np.float64), 3, cfg.C_v).astype(np.float32),
               vertices=spec.vertices.numpy(), cells=spec.cells.numpy(), facets=spec.facets.numpy(),
               period=np.asarray(spec.period), cell_shifts=spec.cell_shifts.numpy(),
               facet_shifts=spec.facet_shifts.numpy(), dim=np.int64(3), n=np.int64(PTILE_N),
               seed=np.int64(PTILE_SEED), tiled_cells=np.int64(len(tcells)))
    out.update(res32)
    out.update({k + "_f64": v for k, v in res64.items()})
    return out


def _fp64_subprocess(case, inputs: dict) -> dict:
    """Run one case's FP64 reference in a fresh process (the dtype shim must precede the import)."""
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
        np.savez(fin, **inputs)
        subprocess.run([sys.executable, os.path.abspath(__file__), "--fp64-worker", case, fin, fout], check=True)
        return dict(np.load(fout))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", action="append")
    ap.add_argument("--fp64-worker", nargs=3, metavar=("CASE", "IN", "OUT"))
    args = ap.parse_args()
    if args.fp64_worker:
        case, fin, fout = args.fp64_worker
        d = np.load(fin)
        if case == "c2dvar":
            res = run_variants(torch.from_numpy(d["prim0"]), float(d["dt"]), fp64=True)
        elif case == "ptile":
            tiled = (d["verts"], d["tcells"], d["facets"], d["mask"], int(d["n_tiles"]))
            res = run_ptile(tiled, d["prim0"], float(d["dt"]), fp64=True)
        else:
            res = run_reference(case, torch.from_numpy(d["prim0"]), float(d["dt"]), fp64=True)
        np.savez(fout, **res)
        return

    from fvm_solver_b200 import meshgen as mg  # noqa: F401
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE))))
    from oracle.fvm_oracle import cfl_dt
    from fvm_solver_b200 import fvm_mesh as fm, tables as tb, config as cf, mesh_store as ms
    for case in args.case or ["c2d", "b3d"]:
        if case in ("c2dvar", "ptile"):
            out = make_variants() if case == "c2dvar" else make_ptile()
            path = os.path.join(HERE, f"fvm_golden_{case}.npz")
            np.savez_compressed(path, **out)
            print(f"wrote {path} ({os.path.getsize(path) / 1e3:.0f} kB)")
            continue
        spec, dim = case_spec(case)
        prim0 = initial_prims(spec, dim)
        cfg = cf.ConfigEllipse()
        if dim == 3:
            cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
            cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
        T = tb.FVMTables(fm.mesh_from_spec(spec), cfg, dim + 2, ms.default_bc_tags(spec.bc_tags, dim))
        from oracle.fvm_oracle import prim_to_state
        U0 = prim_to_state(prim0.numpy().astype(np.float64), dim, cfg.C_v)
        dt = float(cfl_dt(U0, dim, cfg.C_v, cfg.gamma, T.kernel.inv_h.numpy(), 0.5))
        res32 = run_reference(case, prim0, dt, fp64=False)
        with tempfile.TemporaryDirectory() as td:
            fin, fout = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
            np.savez(fin, prim0=prim0.numpy(), dt=dt)
            subprocess.run([sys.executable, os.path.abspath(__file__), "--fp64-worker", case, fin, fout],
                           check=True)
            res64 = dict(np.load(fout))
        out = dict(prim0=prim0.numpy(), dt=np.float64(dt), vertices=spec.vertices.numpy(),
                   cells=spec.cells.numpy(), facets=spec.facets.numpy(),
                   bc_facet_mask=spec.bc_facet_mask.numpy(), bc_tags=np.array(spec.bc_tags),
                   dim=np.int64(dim))
        if case in LIGHT:
            keep32, keep64 = LIGHT[case]
            res32 = {k: res32[k] for k in keep32}
            res64 = {k: res64[k] for k in keep64}
        out.update(res32)
        out.update({k + "_f64": v for k, v in res64.items()})
        path = os.path.join(HERE, f"fvm_golden_{case}.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path} ({os.path.getsize(path) / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
