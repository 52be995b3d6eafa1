"""Generate the golden fixtures by running the reference implementation (CPU path).

Run in a container that has the reference sources (``FVM_REFERENCE_PATH``, default the mounted
reference checkout)::

    python tests/golden/make_golden.py            # writes tests/golden/fvm_golden_<case>.npz

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
"""
from __future__ import annotations

import argparse
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", action="append")
    ap.add_argument("--fp64-worker", nargs=3, metavar=("CASE", "IN", "OUT"))
    args = ap.parse_args()
    if args.fp64_worker:
        case, fin, fout = args.fp64_worker
        d = np.load(fin)
        res = run_reference(case, torch.from_numpy(d["prim0"]), float(d["dt"]), fp64=True)
        np.savez(fout, **res)
        return

    from fvm_solver_b200 import meshgen as mg  # noqa: F401
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE))))
    from oracle.fvm_oracle import cfl_dt
    from fvm_solver_b200 import fvm_mesh as fm, tables as tb, config as cf, mesh_store as ms
    for case in args.case or ["c2d", "b3d"]:
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
