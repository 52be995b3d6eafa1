"""Anchor for the CPU baseline: the reference's own torch CPU path next to the numpy oracle port.

TEST INFRASTRUCTURE ONLY (a timing recipe for the CPU baseline; nothing in the package imports it).

The benchmark's CPU baseline and reference arm time the oracle port (``oracle/fvm_oracle.py``),
because the reference's sources do not travel to the GPU machine.  This script, run where the
reference sources are (``FVM_REFERENCE_PATH``), times both on the same host and the same mesh so
the port's speed relative to the reference is a measured figure:

* the reference: ``FVMEquation.forward`` and one ``Butcher`` RK4 step (``compile=False``, the
  ``SPMGeneral`` torch-sparse CPU operators, ``time_fvm/utils/sparse.py:41-62``) with all host
  threads and with one thread;
* the port: the oracle's residual and RK4 step in one process (one thread), and one
  single-threaded replica per host core run at once (the benchmark's method), aggregated.

The mesh is a non-periodic jittered box (``meshgen.box3d``, the reference has no periodic meshes)
with about as many tetrahedra as the benchmark's CPU sample box; every result is reported per cell.

    FVM_REFERENCE_PATH=<checkout> python oracle/time_reference_cpu.py [--n 21] [--budget 10]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def _timed(fn, budget: float, warm: int = 1) -> tuple:
    for _ in range(warm):
        fn()
    t0, n = time.perf_counter(), 0
    while n < 2 or time.perf_counter() - t0 < budget:
        fn()
        n += 1
    return n, time.perf_counter() - t0


def time_reference(n_box: int, threads: int, budget: float) -> dict:
    import torch
    torch.set_num_threads(threads)
    from refimport import import_reference
    from fvm_solver_b200 import meshgen as mg
    R = import_reference()
    spec = mg.box3d(n_box, seed=4)
    cfg = R["config_fvm"].ConfigEllipse()
    cfg.device, cfg.compile, cfg.plot = "cpu", False, False
    cfg.save_dir = tempfile.mkdtemp(prefix="fvm_cpu_anchor_")
    cfg.solver_name, cfg.solver_extra, cfg.dt = "Butcher", "RK4", 1e-5
    cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
    cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
    st = R["mesh_store"]
    E = st.FacetBCTypes
    bc = {}
    for i, tg in enumerate(spec.bc_tags):
        if tg == "NavierWall":
            bc[i] = st.Facet([E.Dirich] * 3 + [E.Neuman] * 2, [0.0] * 3 + [None, None], [None] * 3 + [0, 0], tag=tg)
        else:
            bc[i] = st.Facet([E.Inlet] * 5, tag=tg)
    t0 = time.perf_counter()
    mesh = R["fvm_mesh"].FVMMesh3D(spec.vertices, spec.cells, spec.facets, spec.bc_facet_mask, device="cpu")
    FE = R["fvm_equation"]
    phy = FE.FluidConstitution3D(cfg, 3)
    N = spec.n_cells
    prim = torch.zeros(N, 5)
    prim[:, 0], prim[:, 3], prim[:, 4] = 3.0, 1.0, 100.0
    prim[:, :3] += 0.1 * torch.randn(N, 3, generator=torch.Generator().manual_seed(0))
    m, r, Q = phy.primatives_to_state(prim[:, :3], prim[:, 3:4], prim[:, 4:])
    eq = FE.FVMEquation(cfg, phy, mesh, 5, bc, us_init=torch.cat([m, r, Q], -1))
    build = time.perf_counter() - t0
    with torch.inference_mode():
        nf, tf = _timed(lambda: eq.forward(prim), budget / 2)
        ns, ts = _timed(lambda: eq.t_solver._solve_step(torch.tensor(0.0)), budget)
    return {"impl": "reference torch CPU (SPMGeneral, compile=False)", "threads": threads, "cells": N,
            "mesh_build_s": build, "forward_ms": 1e3 * tf / nf, "rk4_step_ms": 1e3 * ts / ns,
            "cell_steps_per_s": N * ns / ts}


def _oracle_job(args):
    n_box, budget = args
    import torch
    torch.set_num_threads(1)
    from fvm_solver_b200 import config as cf, fvm_mesh as fm, meshgen as mg, mesh_store as ms, tables as tb
    import fvm_oracle as O
    spec = mg.box3d(n_box, seed=4)
    cfg = cf.ConfigEllipse()
    cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
    cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
    T = tb.FVMTables(fm.mesh_from_spec(spec), cfg, 5, ms.default_bc_tags(spec.bc_tags, 3))
    N = spec.n_cells
    rng = np.random.default_rng(0)
    prim = np.zeros((N, 5), np.float32)
    prim[:, 0], prim[:, 3], prim[:, 4] = 3.0, 1.0, 100.0
    prim[:, :3] += 0.1 * rng.standard_normal((N, 3))
    res = O.OracleResidual(T, cfg, np.float32)
    s = O.OracleSolver(res, O.prim_to_state(prim, 3, cfg.C_v).astype(np.float32), 1e-5)
    nf, tf = _timed(lambda: res.forward(prim), budget / 2)
    ns, ts = _timed(lambda: s.butcher_step("RK4"), budget)
    return N, nf, tf, ns, ts


def time_oracle(n_box: int, budget: float, replicas: int) -> dict:
    os.environ.update(OMP_NUM_THREADS="1", MKL_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    sys.path.insert(0, HERE)
    with mp.get_context("spawn").Pool(replicas) as pool:
        out = pool.map(_oracle_job, [(n_box, budget)] * replicas)
    N = out[0][0]
    one = out[0]
    return {"impl": "numpy oracle port", "replicas": replicas, "cells": N,
            "forward_ms_one_replica": 1e3 * one[2] / one[1], "rk4_step_ms_one_replica": 1e3 * one[4] / one[3],
            "cell_steps_per_s_aggregate": sum(N * ns / ts for _, _, _, ns, ts in out)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=21, help="box3d points per axis (21: ~50k tets)")
    ap.add_argument("--budget", type=float, default=10.0, help="seconds per timed loop")
    args = ap.parse_args()
    cores = os.cpu_count() or 1
    cpu = "unknown CPU"
    try:
        cpu = next((ln.split(":", 1)[1].strip() for ln in open("/proc/cpuinfo") if ln.startswith("model name")), cpu)
    except OSError:
        pass
    ref_all = time_reference(args.n, cores, args.budget)
    ref_one = time_reference(args.n, 1, args.budget)
    orc_one = time_oracle(args.n, args.budget, 1)
    orc_all = time_oracle(args.n, args.budget, cores)
    out = {"host": cpu, "cores": cores, "reference_all_threads": ref_all, "reference_one_thread": ref_one,
           "oracle_one_process": orc_one, "oracle_replicas_all_cores": orc_all,
           "port_over_reference_one_thread": orc_one["cell_steps_per_s_aggregate"] / ref_one["cell_steps_per_s"],
           "port_replicas_over_reference_all_threads":
               orc_all["cell_steps_per_s_aggregate"] / ref_all["cell_steps_per_s"]}
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
