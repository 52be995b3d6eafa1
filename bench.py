#!/usr/bin/env python
"""Benchmark: plain 3D FVM throughput in cell-steps/s on one B200 per rank.

Workload (default): Taylor-Green vortex in a periodic box [0, 2 pi]^3, seeded jittered-grid
Delaunay tetrahedralisation (66^3 points, ~1.96 M tetrahedra, jitter 0.2 h), Mach 0.1, Re 1600,
FP32 5-variable state, classic RK4 with a CFL 0.5 time step recomputed on the device every step.
A "step" is one full RK4 step (4 residual evaluations + stage updates + FP64 CFL reduction).

* ``value``  -- cell-steps/s of the whole job: sum over ranks of cells x K / max over ranks of
  the device time of K steps replayed from a CUDA graph (W eager warm-up steps and one untimed
  replay of the graph first; inputs resident in HBM; the per-stage working set, >1 GB, is larger
  than L2, so no L2 flush is needed).
* ``e2e``    -- the same metric through the public API with host buffers: ``TSolver.step_host``
  advances max(K, 50) independent pinned host states (a ring of 4 distinct snapshots) by one
  step each: every step copies its state host->device, restarts the solver on it (CFL time step
  from the state, no carried gradients), steps, and copies the result back (the device part as
  one CUDA-graph replay); the copies run on two copy streams and overlap the neighbouring steps.  ``chained_value`` is the serial case where each
  step's input is the previous step's output read back to the host (nothing can overlap).
  ``bound`` sets the streamed step time against the slower of one state's device work (its
  graph replayed alone: copy into the state, restart, step, copy out) and one state copied in
  and one out at the same time (timed alone): ``frac`` = that bound / the step time.
* ``roofline`` -- the dominant kernel's algorithmic bytes per launch / its mean CUDA-event
  duration over a second timed pass of K steps (events bracket every launch), against the
  measured HBM copy bandwidth.
* ``cpu_baseline`` -- the numpy oracle (a restatement of the reference's CPU path) timed on this
  host for a bounded sample (a 20^3-point periodic box).

``--impl reference`` times that oracle port alone (the reference is Python and cannot run here).
Multi-GPU (torchrun): each rank advances its own box (different seed); no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=66, help="points per axis of the periodic box")
    ap.add_argument("--sample-n", type=int, default=20, help="points per axis of the CPU sample box")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--train-cases", type=int, default=None, help="corrector: 32 (2D) / 4 (3D)")
    ap.add_argument("--eval-cases", type=int, default=16)
    ap.add_argument("--iters", type=int, default=None, help="corrector training iterations: 6000 (2D) / 2000 (3D)")
    ap.add_argument("--drift-steps", type=int, default=500,
                    help="channel_cylinder: steps of the trajectory compared with the FP32/FP64 oracle (0: skip)")
    ap.add_argument("--parts", type=int, default=4,
                    help="partitioned workload on one GPU: parts the box is split into")
    ap.add_argument("--windows", type=int, default=50, help="corrector rollout windows of k = 8 steps")
    ap.add_argument("--checkpoint", default=None, help="corrector: evaluate this stored model (no training)")
    ap.add_argument("--cases-per-batch", type=int, default=0,
                    help="corrector: stream the training cases in batches of this many meshes (0: one batch)")
    ap.add_argument("--record-steps", type=int, default=100, help="corrector streaming: steps recorded per batch")
    ap.add_argument("--gates", default=None,
                    help="corrector acceptance gates, 'ratio[:consistency],...' (first one is the headline)")
    ap.add_argument("--save-checkpoint", default=None, help="corrector: save the trained model here")
    ap.add_argument("--workload", default="taylor_green",
                    choices=["taylor_green", "channel_cylinder", "ensemble", "corrector", "corrector3d",
                             "partitioned"],
                    help="taylor_green: the headline 3D box; channel_cylinder: the 2D cylinder case (11k cells); "
                         "ensemble: batched 2D ensemble vs the same cases run one by one")
    ap.add_argument("--cases", type=int, default=256, help="ensemble size")
    ap.add_argument("--ensemble-cfl", type=float, default=None, help="ensemble: CFL of the fixed per-case dt")
    ap.add_argument("--launch", default=None,
                    help="fixed block sizes instead of the autotuner, e.g. cell=128,face=128,div_stage=64")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline line without the channel / ensemble / corrector keys")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def _oracle_channel_trajectory(job):
    """The oracle's SSP-RK3 + CFL 0.5 run of the channel-cylinder case from its initial condition,
    in float32 or float64; returns the conserved state every ``every`` steps."""
    dtype_name, n_steps, every = job
    torch.set_num_threads(1)
    from fvm_solver_b200 import workloads as W
    from oracle import fvm_oracle as O
    dt_ = np.float32 if dtype_name == "f32" else np.float64
    case = W.channel_cylinder(device="cpu")
    T = case.tables()
    res = O.OracleResidual(T, case.cfg, dt_)
    inv_h = T.kernel.inv_h.numpy()
    s = O.OracleSolver(res, case.state0.numpy().astype(dt_), 1e-4)
    out = []
    for k in range(1, n_steps + 1):
        s.dt = res.dt(O.cfl_dt(s.state, 2, case.cfg.C_v, case.cfg.gamma, inv_h, 0.5))
        s.butcher_step("SSP_RK3")
        if k % every == 0:
            out.append(np.asarray(s.state, dtype=np.float64).copy())
    return out


def channel_drift(n_steps: int, every: int = 100) -> dict:
    """Config-1 trajectory agreement: the CUDA path's state after 100, 200, ... SSP-RK3 steps
    against the FP32 oracle (the reference's arithmetic) and the FP64 oracle, as rel-L2 over the
    whole state (a drift curve; the flow is unsteady, so differences grow with time)."""
    import multiprocessing as mp
    from fvm_solver_b200 import workloads as W
    with mp.get_context("spawn").Pool(2) as pool:
        pending = pool.map_async(_oracle_channel_trajectory, [("f32", n_steps, every), ("f64", n_steps, every)])
        case = W.channel_cylinder(device="cuda")
        eq = case.equation()
        gpu = []
        for k in range(1, n_steps + 1):
            eq.t_solver.step(1)
            if k % every == 0:
                gpu.append(eq.cells.state.double().cpu().numpy())
        o32, o64 = pending.get()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return {"steps": list(range(every, n_steps + 1, every)),
            "gpu_vs_oracle_fp32": [rel(g, o) for g, o in zip(gpu, o32)],
            "gpu_vs_oracle_fp64": [rel(g, o) for g, o in zip(gpu, o64)],
            "oracle_fp32_vs_fp64": [rel(a, b) for a, b in zip(o32, o64)]}


def _oracle_worker(job):
    """One single-threaded oracle replica: (cells, steps done, seconds) of RK4 + CFL steps on the
    sample box after ``warmup`` untimed steps; ``steps`` fixed, or as many as fit ``budget_s``."""
    sample_n, steps, warmup, budget_s = job
    torch.set_num_threads(1)
    from fvm_solver_b200 import workloads as W
    from oracle import fvm_oracle as O
    case = W.taylor_green(n=sample_n, seed=0, device="cpu")
    T = case.tables()
    res = O.OracleResidual(T, case.cfg, np.float32)
    state = case.state0.numpy()
    inv_h = T.kernel.inv_h.numpy()
    s = O.OracleSolver(res, state, O.cfl_dt(state, 3, case.cfg.C_v, case.cfg.gamma, inv_h, 0.5))

    def step():
        s.dt = res.dt(O.cfl_dt(s.state, 3, case.cfg.C_v, case.cfg.gamma, inv_h, 0.5))
        s.butcher_step("RK4")

    for _ in range(warmup):
        step()
    t0, n = time.perf_counter(), 0
    while (steps is None and time.perf_counter() - t0 < budget_s) or (steps is not None and n < steps):
        step()
        n += 1
    return case.spec.n_cells, n, time.perf_counter() - t0


def cpu_replicas(sample_n: int, steps: int | None = None, warmup: int = 1, budget_s: float = 15.0) -> dict:
    """The oracle (numpy restatement of the reference's CPU path) on every host core: one
    single-threaded replica of the sample box per core (spawned processes, capped so that each has
    ~1 GB of free memory), aggregate cell-steps/s.  Independent replicas are an upper bound of what
    one multi-threaded run of the reference's torch CPU path reaches on the same cores."""
    import multiprocessing as mp
    import psutil
    workers = max(1, min(os.cpu_count() or 1, int(psutil.virtual_memory().available * 0.5 // 1e9)))
    saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "MKL_NUM_THREADS", "OPENBLAS_NUM_THREADS")}
    for k in saved:
        os.environ[k] = "1"
    try:
        with mp.get_context("spawn").Pool(workers) as pool:
            out = pool.map(_oracle_worker, [(sample_n, steps, warmup, budget_s)] * workers)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    N = out[0][0]
    value = sum(n_ * k / el for n_, k, el in out)
    el_max = max(el for _, _, el in out)
    k_min = min(k for _, k, _ in out)
    cpu_model = "unknown CPU"
    try:
        with open("/proc/cpuinfo") as fh:
            cpu_model = next((ln.split(":", 1)[1].strip() for ln in fh if ln.startswith("model name")), cpu_model)
    except OSError:
        pass
    return {"value": value, "unit": "cell-steps/s", "cores": workers, "kind": "port",
            "sample": f"{workers} single-threaded numpy oracle replicas ({cpu_model}), periodic TGV box "
                      f"{sample_n}^3 points ({N} tets) each, >= {k_min} RK4 steps each in {el_max:.1f} s",
            "ms_per_step": 1e3 * el_max / max(k_min, 1), "anchor": cpu_anchor()}


def cpu_anchor():
    """How fast the port runs next to the reference's own torch CPU path on one host
    (``oracle/cpu_anchor.json``, measured by ``oracle/time_reference_cpu.py`` where the reference
    sources are): the port's all-core throughput over the reference's all-thread throughput."""
    p = os.path.join(ROOT, "oracle", "cpu_anchor.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return {"port_over_reference_all_threads": d["port_replicas_over_reference_all_threads"],
            "port_over_reference_one_thread": d["port_over_reference_one_thread"],
            "host": d["host"], "source": "oracle/cpu_anchor.json"}


def cpu_baseline(sample_n: int, budget_s: float = 15.0):
    """CPU baseline of the benchmark line: the oracle on every host core for ~budget_s."""
    return cpu_replicas(sample_n, steps=None, warmup=1, budget_s=budget_s)


def parity_check(sample_n: int, steps: int = 5) -> dict:
    """The CUDA path vs the oracle on the sample box: rel-L2 of the state after ``steps`` RK4 + CFL
    steps against the FP32 oracle (the reference's arithmetic) and the FP64 oracle."""
    from fvm_solver_b200 import workloads as W
    from oracle import fvm_oracle as O
    case = W.taylor_green(n=sample_n, seed=0, device="cuda")
    eq = case.equation()
    eq.t_solver.step(steps)
    got = eq.cells.state.double().cpu().numpy()
    T = eq.tables
    inv_h = T.kernel.inv_h.numpy()
    out = {"steps": steps, "cells": case.spec.n_cells}
    for name, dt in (("fp32", np.float32), ("fp64", np.float64)):
        res = O.OracleResidual(T, case.cfg, dt)
        s = O.OracleSolver(res, case.state0.numpy().astype(dt), 1.0)
        for _ in range(steps):
            s.dt = res.dt(O.cfl_dt(s.state, 3, case.cfg.C_v, case.cfg.gamma, inv_h, 0.5))
            s.butcher_step("RK4")
        ref = s.state.astype(np.float64)
        out[f"rel_l2_vs_oracle_{name}"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return out


def run_reference(args):
    """The reference arm: the oracle port of the reference's CPU path on every host core (see
    ``cpu_replicas``), warm-up + K RK4 steps per replica; rank 0 alone under torchrun."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cpu = cpu_replicas(args.sample_n, steps=args.steps, warmup=args.warmup)
    v = cpu["value"]
    out = {"impl": "reference", "metric": "cell-steps/s", "value": v, "unit": "cell-steps/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "taylor_green_periodic_box_rk4_cfl0.5", "sample_points_per_axis": args.sample_n},
           "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "anchor")},
           "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def partitioned_bench(args):
    """One Taylor-Green box split into parts with one-cell halos (``fvm_solver_b200.partition``).

    One process (no torchrun): ``--parts`` parts stepped on one GPU, exchanges as device copies;
    reports the partitioned throughput next to the unpartitioned one on the same box and checks the
    two final states (after a warm-up replay and a timed replay of K steps each) for bitwise equality.  Under torchrun (N > 1): one part per rank, halo rows over
    NCCL point-to-point, FP64 reductions over NCCL all-reduce; strong scaling (the box is fixed).
    """
    import torch.distributed as dist
    from fvm_solver_b200 import workloads as W
    from fvm_solver_b200.autotune import autotune
    from fvm_solver_b200.partition import DistComm, LocalComm, PartitionedSolver, split_tables
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    case = W.taylor_green(n=args.n, device=f"cuda:{local}")
    eq = case.equation()
    autotune(eq)
    N = eq.mesh.n_cells
    state0 = eq.cells.state.clone()
    t0 = time.time()
    P = world if world > 1 else args.parts
    parts = split_tables(eq.tables.kernel, P)
    t_split = time.time() - t0
    R, G = eq.dev.row, eq.dev.grow
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        ps = PartitionedSolver([parts[rank]], DistComm(parts[rank], f"cuda:{local}"), eq.phys, eq.t_solver.tab,
                               device=f"cuda:{local}")
        ps.set_state(state0)
        ps.cfl_dt(case.cfg.cfl)
        ps.step(args.warmup)
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ps.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        halo = torch.tensor([ps.halo_rows()], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(halo)
        dist.barrier()
        dist.destroy_process_group()
        if rank == 0:
            ms = float(t.item())
            print(json.dumps({"metric": "cell-steps/s", "value": N * args.steps / (ms / 1e3), "unit": "cell-steps/s",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                              "dtype": "f32", "data": "synthetic",
                              "config": {"workload": "taylor_green_partitioned", "cells": N, "parts": world,
                                         "halo_rows_total": int(halo.item()),
                                         "exchange": "NCCL point-to-point halo rows, NCCL all-reduce"}}))
        return
    # one GPU: single mesh, then the same box in P parts, both from state0 for K graph-replayed steps
    sol = eq.t_solver
    replay = sol.graph_steps(args.steps)
    replay()                                 # untimed warm-up replay (uploads the graph)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    replay()
    b.record(stream)
    torch.cuda.synchronize()
    ms_single = a.elapsed_time(b)
    want = eq.cells.state.clone()
    del replay
    ps = PartitionedSolver(parts, LocalComm(parts, "cuda"), eq.phys, sol.tab)
    ps.set_state(state0)
    ps.cfl_dt(case.cfg.cfl)
    preplay = ps.graph_steps(args.steps)
    preplay()                                # untimed warm-up replay: both runs end after 2 K steps
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        a.record(stream)
        preplay()
        b.record(stream)
        torch.cuda.synchronize()
    ms_part = a.elapsed_time(b)
    got = torch.empty_like(want)
    ps.gather_state(got)
    halo = ps.halo_rows()
    stages = sol.tab.stages
    print(json.dumps({"metric": "cell-steps/s", "value": N * args.steps / (ms_part / 1e3), "unit": "cell-steps/s",
                      "n_gpus": 1, "steps": args.steps, "warmup": 0, "ms_per_step": ms_part / args.steps,
                      "higher_is_better": True, "dtype": "f32", "data": "synthetic",
                      "config": {"workload": "taylor_green_partitioned_on_one_gpu", "cells": N, "parts": P,
                                 "timing": "cuda graph replay", "split_seconds": t_split},
                      "unpartitioned": {"value": N * args.steps / (ms_single / 1e3), "ms_per_step": ms_single / args.steps},
                      "halo_rows_total": halo, "halo_fraction": halo / N,
                      "exchange_bytes_per_step": halo * 4 * (R + G) * stages,
                      "bitwise_equal_to_unpartitioned": bool(torch.equal(got, want)),
                      "clocks": clk.summary()}))


def graph_timer(stream):
    """Device time (ms) of K steps replayed from one CUDA graph, after an untimed upload replay."""
    def timed(sol, steps):
        replay = sol.graph_steps(steps)
        replay()                             # untimed: the first replay also uploads the graph
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        replay()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    return timed


def channel_cylinder_result(steps: int, warmup: int, drift_steps: int, cpu: bool, timed) -> dict:
    """Config 1: the 2D channel-cylinder case (11 323 triangles), SSP-RK3 at CFL 0.5, cell-steps/s
    from a graph replay of ``steps`` steps; the CPU oracle on the same mesh (1 core, ~15 s); the
    ``drift_steps``-step trajectory against the FP32 and FP64 oracle."""
    from fvm_solver_b200 import workloads as W
    from fvm_solver_b200.autotune import autotune, tune_fused
    case = W.channel_cylinder(device="cuda")
    eq = case.equation()
    sol = eq.t_solver
    autotune(eq)
    fused = tune_fused(eq)
    sol.step(warmup)
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = timed(sol, steps)
    N = eq.mesh.n_cells
    cpu_out = None
    if cpu:
        from oracle import fvm_oracle as O
        T = eq.tables
        res = O.OracleResidual(T, case.cfg, np.float32)
        s = O.OracleSolver(res, case.state0.numpy(), 1e-4)
        inv_h = T.kernel.inv_h.numpy()
        t0, n = time.perf_counter(), 0
        while time.perf_counter() - t0 < 15.0:
            s.dt = res.dt(O.cfl_dt(s.state, 2, case.cfg.C_v, case.cfg.gamma, inv_h, 0.5))
            s.butcher_step("SSP_RK3")
            n += 1
        el = time.perf_counter() - t0
        cpu_out = {"value": N * n / el, "unit": "cell-steps/s", "cores": 1, "kind": "port",
                   "sample": f"numpy oracle, same mesh ({N} cells), {n} SSP-RK3 steps, {el:.1f} s"}
    drift = channel_drift(drift_steps) if drift_steps else None
    return {"metric": "cell-steps/s", "value": N * steps / (ms / 1e3), "unit": "cell-steps/s",
            "steps": steps, "warmup": warmup, "ms_per_step": ms / steps, "dtype": "f32",
            "config": {"workload": "channel_cylinder_2d_ssprk3_cfl0.5", "cells": N, "facets": eq.dev.n_facets,
                       "l2": "working set fits in L2 (launch/latency bound case)", "timing": "cuda graph replay",
                       "step": "fused (one cooperative launch per step)" if fused["fused"] else "separate launches",
                       "ms_per_step_by_variant": fused["ms_per_step"]},
            "cpu_baseline": cpu_out, "drift_vs_oracle": drift, "clocks": clk.summary()}


ENSEMBLE_CFL = 0.3


def ensemble_result(cases: int, steps: int, warmup: int, timed, cfl: float = ENSEMBLE_CFL) -> dict:
    """Config 3: 256 seeded channel-cylinder cases (2k-60k cells each) advanced by one launch per
    kernel (AB3 after two SSP-RK3 start-up steps), against the same cases run one after another,
    each with its own CUDA graph, autotuned block sizes and its faster step form."""
    from fvm_solver_b200 import batched as B, workloads as W
    from fvm_solver_b200.autotune import autotune, tune_fused
    from fvm_solver_b200.equation import FVMEquation, FluidConstitution2D
    t0 = time.time()
    parts = B.build_ensemble_tables(cases, workers=min(16, os.cpu_count() or 1))
    t_build = time.time() - t0
    cfg = W.ensemble_case(0, device="cuda", cfl=cfl).cfg
    batch = B.BatchedFVM(parts, cfg, device="cuda")
    Nt = batch.n_cells
    tuned = {k: v["threads"] for k, v in autotune(batch).items()}
    batch.t_solver.step(max(warmup, 3))
    fused_b = tune_fused(batch)
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms_b = timed(batch.t_solver, steps)
    finite = bool(torch.isfinite(batch.cells.state).all())
    roof = batched_roofline(batch, steps=10)
    del batch
    torch.cuda.empty_cache()
    ms_p, cells_p, n_fused = 0.0, 0, 0
    for k, p in enumerate(parts):
        c = W.ensemble_case(k, device="cuda", cfl=cfl).cfg
        eq = FVMEquation.from_kernel_tables(c, FluidConstitution2D(c), p.kt, p.state0)
        autotune(eq)                       # per size bucket (cached), so small cases get their own
        eq.t_solver.step(max(warmup, 3))
        n_fused += tune_fused(eq)["fused"]  # each case alone also gets its faster step form
        ms_p += timed(eq.t_solver, steps)
        cells_p += p.kt.n_cells
        del eq
    vb = Nt * steps / (ms_b / 1e3)
    vp = cells_p * steps / (ms_p / 1e3)
    sizes = [p.kt.n_cells for p in parts]
    return {"metric": "cell-steps/s", "value": vb, "unit": "cell-steps/s", "steps": steps, "warmup": warmup,
            "ms_per_step": ms_b / steps, "dtype": "f32",
            "config": {"workload": "ensemble_2d_ab3_batched", "cases": cases, "cells_total": Nt,
                       "cells_min": min(sizes), "cells_max": max(sizes),
                       "integrator": f"AB3 (SSP-RK3 start), fixed per-case dt from CFL {cfl} at the start",
                       "cfl_note": ENSEMBLE_CFL_NOTE if cfl != 0.5 else None,
                       "timing": "cuda graph replay", "table_build_s": t_build, "host_cpus": os.cpu_count(),
                       "block_sizes": tuned, "fused_step": fused_b},
            "state_finite_after_timed_steps": finite,
            "roofline": roof,
            "plain": {"value": vp, "unit": "cell-steps/s", "ms_per_step_all_cases": ms_p / steps,
                      "how": "each case alone, own CUDA graph, sequential",
                      "cases_with_fused_step": n_fused},
            "batched_over_plain": vb / vp, "clocks": clk.summary()}


ENSEMBLE_CFL_NOTE = ("AB3 with a time step fixed at the start: CFL 0.3 keeps every case inside AB3's "
                     "stability region for 2000 steps; see DESIGN section 5")


def ensemble_sharded(args):
    """The ensemble under torchrun: cases split across the ranks by cell count
    (``sharding.partition_cases``), one ``BatchedFVM`` per rank, no collective in the step, the
    graph-replayed steps timed on each rank's device and reduced with MAX; one all-gather of the
    per-case results (cells, final dt, sum of the state, finite flag) at the end.  The total work
    is fixed as ranks are added (strong scaling)."""
    import torch.distributed as dist
    from datetime import timedelta
    from fvm_solver_b200 import batched as B, workloads as W
    from fvm_solver_b200.autotune import autotune
    from fvm_solver_b200.sharding import run_sharded
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    rank, world = dist.get_rank(), dist.get_world_size()
    cfl = args.ensemble_cfl or ENSEMBLE_CFL
    sizes = [p["n_cells"] for p in (W.ensemble_params(i) for i in range(args.cases))]
    stream = torch.cuda.current_stream()
    timed = graph_timer(stream)
    dev = torch.device("cuda", local)
    holder = {}

    def make_batch(ids):
        if not ids:
            return None
        workers = max(1, min(16, (os.cpu_count() or 1) // world))
        parts = B.build_ensemble_tables(args.cases, workers=workers, indices=ids)
        cfg = W.ensemble_case(ids[0], device=f"cuda:{local}", cfl=cfl).cfg
        batch = B.BatchedFVM(parts, cfg, device=f"cuda:{local}")
        holder["tuned"] = {k: v["threads"] for k, v in autotune(batch).items()}
        batch.t_solver.step(max(args.warmup, 3))
        return batch

    def advance(batch, steps):
        with ClockSampler(local) as clk:
            ms = timed(batch.t_solver, steps)
        holder["clocks"] = clk.summary()
        return ms

    def rows(batch):
        out = []
        for k in range(batch.n_cases):
            st = batch.case_state(k)
            out.append(torch.stack([torch.tensor(float(st.shape[0]), device=dev, dtype=torch.float64),
                                    batch.t_solver.dt[k].double(), st.double().sum(),
                                    torch.isfinite(st).all().double()]))
        return torch.stack(out)

    res = run_sharded(sizes, args.steps, make_batch, advance, rows, row_width=4, device=dev)
    table = res["rows"].cpu()
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        ms = res["ms_max"]
        print(json.dumps({"metric": "cell-steps/s", "value": res["cells_total"] * args.steps / (ms / 1e3),
                          "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                          "dtype": "f32", "data": "synthetic",
                          "config": {"workload": "ensemble_2d_ab3_batched_sharded", "cases": args.cases,
                                     "cells_total": res["cells_total"], "cells_rank0": res["cells_local"],
                                     "integrator": f"AB3 (SSP-RK3 start), fixed per-case dt from CFL {cfl}",
                                     "sharding": "cases by cell count (LPT), one BatchedFVM per rank, "
                                                 "no collective in the step; one all-gather of results",
                                     "block_sizes_rank0": holder.get("tuned"), "timing": "cuda graph replay, "
                                     "max over ranks"},
                          "cases_finite": int(table[:, 3].sum().item()), "clocks": holder.get("clocks")}))


def secondary(args):
    """Secondary workloads (single GPU) as their own benchmark lines."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dp_training = args.workload in ("corrector", "corrector3d") and args.cases_per_batch and not args.checkpoint
    if world > 1 and args.workload not in ("partitioned", "ensemble") and not dp_training:
        sys.exit(f"--workload {args.workload} runs on one GPU; several ranks run the default workload "
                 f"(one box per rank), --workload ensemble (cases split across the ranks), "
                 f"--workload partitioned (one box split across the ranks) or corrector training with "
                 f"--cases-per-batch (data-parallel)")
    if world > 1 and dp_training:
        return corrector_bench_dp(args)
    if args.workload == "partitioned":
        return partitioned_bench(args)
    if args.workload == "ensemble" and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        return ensemble_sharded(args)
    torch.cuda.set_device(0)
    timed = graph_timer(torch.cuda.current_stream())
    if args.workload in ("corrector", "corrector3d"):
        return corrector_bench(args, timed)
    common = {"n_gpus": 1, "higher_is_better": True, "data": "synthetic"}
    if args.workload == "channel_cylinder":
        out = channel_cylinder_result(args.steps, args.warmup, args.drift_steps, not args.no_cpu_baseline, timed)
    else:
        out = ensemble_result(args.cases, args.steps, args.warmup, timed, cfl=args.ensemble_cfl or ENSEMBLE_CFL)
    print(json.dumps({**out, **common}))


def batched_roofline(batch, steps: int = 10) -> dict:
    """Per-kernel achieved bandwidth of the batched AB3 step (an eager pass of ``steps`` steps with
    every launch bracketed by CUDA events): algorithmic bytes (``roofline.kernel_bytes``; the
    Adams step's divergence kernel reads two stored increments and writes one plus the state) over
    the mean launch time, against the measured HBM copy bandwidth."""
    from fvm_solver_b200 import _lib
    from fvm_solver_b200.roofline import kernel_bytes
    lib = _lib.load()
    kt = batch.kt
    _lib.check(lib.fvm_profile_start(steps * 16 + 16), "fvm_profile_start")
    batch.t_solver.step(steps)
    n = lib.fvm_profile_stop()
    torch.cuda.synchronize()
    ids = np.zeros(max(n, 1), np.int32)
    ms = np.zeros(max(n, 1), np.float32)
    if n <= 0 or lib.fvm_profile_read(n, ids.ctypes.data, ms.ctypes.data) != n:
        return None
    kb = kernel_bytes(kt.dim, kt.n_cells, kt.n_facets, kt.n_bc)
    byts = {"bc": kb["bc"], "cell": kb["cell"], "face": kb["face"], "div_stage": kb["div_base"] + 4 * kb["row"]}
    peak, peak_kind = measured_peaks()
    kern = {}
    for kid, name in ((2, "bc"), (3, "cell"), (4, "face"), (5, "div_stage")):
        sel = ids == kid
        if not np.any(sel):
            continue
        m = float(ms[sel].mean())
        kern[name] = {"ms_mean": m, "share": float(ms[sel].sum() / ms[:n].sum()),
                      "algorithmic_bytes_per_launch": byts[name], "achieved_gbs": byts[name] / (m / 1e3) / 1e9}
    dom = max(kern, key=lambda k: kern[k]["share"])
    return {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
            "frac": kern[dom]["achieved_gbs"] / peak, "peak_source": peak_kind, "kernels": kern}


CORRECTOR_CKPT = os.path.join(ROOT, "fvm_solver_b200", "checkpoints", "corrector_2d_k8.pt")


def _corrector_family(three_d: bool):
    from fvm_solver_b200 import workloads as W
    params = (lambda i, seed: W.sphere_params(i, seed)) if three_d else W.ensemble_params
    seeds = (5678, 9100) if three_d else (1234, 9000)
    return params, seeds


def _corrector_cases(n, seed, three_d):
    """Tables, solver config (SSP-RK3, dt fixed per case from CFL 0.5 at the start) and per-case
    (Mach, log10 Re) of ``n`` seeded cases of the channel (2D) or sphere (3D) family."""
    import copy
    from fvm_solver_b200 import batched as B, workloads as W
    params, _ = _corrector_family(three_d)
    parts = B.build_ensemble_tables(n, base_seed=seed, workers=min(16, os.cpu_count() or 1),
                                    family="sphere" if three_d else "channel")
    case0 = W.sphere_case(0, device="cuda", base_seed=seed, cells=(20_000, 20_000)) if three_d else \
        W.ensemble_case(0, device="cuda", base_seed=seed)
    cfg = copy.deepcopy(case0.cfg)
    cfg.solver_name, cfg.solver_extra, cfg.cfl = "Butcher", "SSP_RK3", None
    prm = torch.tensor([[params(i, seed)["mach"], np.log10(params(i, seed)["reynolds"])] for i in range(n)],
                       dtype=torch.float32)
    return parts, cfg, prm


def host_memory() -> str:
    """Available host memory and this process's resident size, for the training log."""
    try:
        import psutil
        return (f"host available {psutil.virtual_memory().available / 2**30:.1f} GiB, "
                f"rss {psutil.Process().memory_info().rss / 2**30:.1f} GiB")
    except Exception:                                    # psutil missing: no figures
        return "host memory n/a"


def corrector_train_streaming(args, three_d: bool, group=None):
    """Config 4 scale: ``args.train_cases`` seeded cases in batches of ``args.cases_per_batch``
    meshes (a batch's tables are built by a pool of host processes while the GPU trains on the
    previous batch), ``args.iters`` Adam iterations in all (``corrector.train_streaming``).  With a
    process group of W ranks, training is data-parallel: rank r streams the global batches
    r, r + W, r + 2W, ... (the cases are split, not repeated) and every iteration averages the
    gradients of all ranks, so each iteration sees W batches of cases."""
    import copy
    from fvm_solver_b200 import batched as B, workloads as W
    from fvm_solver_b200.corrector import train_streaming
    params, seeds = _corrector_family(three_d)
    family = "sphere" if three_d else "channel"
    per = args.cases_per_batch
    import torch.distributed as dist
    world = dist.get_world_size(group) if group is not None or dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    n_batches = max(1, args.train_cases // per // world)
    case0 = W.sphere_case(0, device="cuda", base_seed=seeds[0], cells=(20_000, 20_000)) if three_d else \
        W.ensemble_case(0, device="cuda", base_seed=seeds[0])
    cfg = copy.deepcopy(case0.cfg)
    cfg.solver_name, cfg.solver_extra, cfg.cfl = "Butcher", "SSP_RK3", None
    workers = max(1, min(12, (os.cpu_count() or 2) - 2))
    state = {}
    pool = B.TableWorkers(workers)
    queued = set()

    def cases_of(b):                                     # local batch b -> global batch b W + r
        gb = b * world + rank
        return range(gb * per, (gb + 1) * per)

    def prefetch(b):
        if b not in queued:
            for i in cases_of(b):
                pool.submit(i, (i, seeds[0], family, (300_000, 800_000)))
            queued.add(b)

    def make_batch(b):
        prefetch(b)
        parts = [pool.get(i) for i in cases_of(b)]
        queued.discard(b)
        batch = B.BatchedFVM(parts, cfg, device="cuda")
        batch.t_solver.update_cfl_dt(0.5)
        prm = torch.tensor([[params(i, seeds[0])["mach"], np.log10(params(i, seeds[0])["reynolds"])]
                            for i in cases_of(b)], dtype=torch.float32)
        return batch, prm

    def log(b, done, cases, loss):
        if rank == 0 and (b % max(1, n_batches // 20) == 0 or b == n_batches - 1):
            print(f"batch {b + 1}/{n_batches}: {done} iterations, {cases} cases, loss {loss:.4g}, "
                  f"{time.time() - t0:.0f} s; {host_memory()}; table workers replaced {pool.restarts} "
                  f"(exit codes {sorted(set(pool.exit_codes))})", file=sys.stderr, flush=True)
        if save_every and (b + 1) % save_every == 0 and args.save_checkpoint and rank == 0:
            state["model"].save(args.save_checkpoint + ".partial", meta={"batches_done": b + 1, "iters_done": done})

    save_every = max(1, n_batches // 10)
    t0 = time.time()
    try:
        model, hist, cases = train_streaming(make_batch, n_batches, args.iters, k=8, record=args.record_steps,
                                             spinup=200, prefetch=prefetch, log=log, keep=state, group=group)
    finally:
        pool.close()
    torch.cuda.synchronize()
    info = {"train_cases": cases * world, "cases_per_batch": per, "batches": n_batches * world, "iters": args.iters,
            "table_workers": workers, "worker_restarts": pool.restarts,
            "worker_exit_codes": sorted(set(pool.exit_codes)), "data_parallel_ranks": world,
            "recorded_steps_per_case": args.record_steps + 8, "loss_first": hist[0][1], "loss_last": hist[-1][1],
            "loss_history": hist[:: max(1, len(hist) // 20)], "seconds": time.time() - t0}
    return model, info


def corrector_train(args, three_d: bool):
    """Train the corrector on trajectories of ``args.train_cases`` seeded cases; returns the model
    and a summary (loss history, seconds)."""
    if args.cases_per_batch:
        return corrector_train_streaming(args, three_d)
    from fvm_solver_b200 import batched as B
    from fvm_solver_b200.corrector import CorrectorModel, record_trajectory, train
    _, seeds = _corrector_family(three_d)
    t0 = time.time()
    parts, cfg, prm = _corrector_cases(args.train_cases, seeds[0], three_d)
    batch = B.BatchedFVM(parts, cfg, device="cuda")
    batch.t_solver.update_cfl_dt(0.5)
    traj = record_trajectory(batch, steps=200 if three_d else 400, spinup=200)
    model = CorrectorModel(batch, prm, k=8, seed=0, lr=1e-3)
    torch.cuda.synchronize()
    t1 = time.time()
    hist = train(model, traj, iters=args.iters, log_every=max(1, args.iters // 10))
    torch.cuda.synchronize()
    info = {"train_cases": args.train_cases, "train_cells": int(batch.n_cells), "iters": args.iters,
            "loss_first": hist[0][1], "loss_last": hist[-1][1], "seconds": time.time() - t1,
            "setup_seconds": t1 - t0}
    del traj
    torch.cuda.empty_cache()
    return model, info


CORRECTOR_GATES = ((3.0, 0.0), (1.2, 0.0), (3.0, 0.5), (3.0, 0.3), (1.5, 0.3))


def parse_gates(text: str | None) -> tuple:
    """"3.0,1.2:0.3" -> ((3.0, 0.0), (1.2, 0.3)): residual ratio[:trapezoid consistency] per gate."""
    if not text:
        return CORRECTOR_GATES
    out = []
    for item in text.split(","):
        r, _, c = item.partition(":")
        out.append((float(r), float(c) if c else 0.0))
    return tuple(out)


def corrector_evaluate(model_src, args, three_d: bool, gates=None, spinup: int = 200) -> dict:
    """Held-out cases advanced ``args.windows`` windows of k = 8 steps (a) by plain FVM (a CUDA graph
    of 8 steps per window) and (b) by the corrector with per-case checks and FVM fallback (the
    proposal + checks graph, one host read of the verdicts, the 8-step graph for failed cases), both
    from the same spun-up start and timed with CUDA events; the corrected states are compared with
    the plain ones at the end.  ``model_src``: a trained model, or a checkpoint path.  ``gates``:
    (residual ratio, trapezoid consistency or 0) per rollout; the first is the line's headline."""
    gates = parse_gates(getattr(args, "gates", None)) if gates is None else gates
    from fvm_solver_b200 import batched as B
    from fvm_solver_b200.corrector import CheckedRollout, CorrectorModel
    _, seeds = _corrector_family(three_d)
    eparts, ecfg, eprm = _corrector_cases(args.eval_cases, seeds[1], three_d)
    stream = torch.cuda.current_stream()
    plain = B.BatchedFVM(eparts, ecfg, device="cuda")
    plain.t_solver.update_cfl_dt(0.5)
    plain.t_solver.step(spinup)
    plain_window = plain.t_solver.graph_steps(8)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e[0].record(stream)
        for _ in range(args.windows):
            plain_window()
        e[1].record(stream)
        torch.cuda.synchronize()
    ms_plain = e[0].elapsed_time(e[1])
    n_cases = args.eval_cases
    curve_at = [w for w in (10, 25, 50, 100, 250, 500, 1000) if w <= args.windows]

    def case_rel(a_state, b_state, batch) -> torch.Tensor:
        """Per-case rel-L2 of a_state against b_state (FP64)."""
        cc = batch.dev.case["cell_case"].long()
        d = torch.zeros(n_cases, dtype=torch.float64, device=a_state.device)
        r = torch.zeros_like(d)
        d.index_add_(0, cc, (a_state.double() - b_state.double()).square().sum(1))
        r.index_add_(0, cc, b_state.double().square().sum(1))
        return (d / r).sqrt()

    def make_corr():
        corr = B.BatchedFVM(eparts, ecfg, device="cuda")
        corr.t_solver.update_cfl_dt(0.5)
        corr.t_solver.step(spinup)
        model = CorrectorModel.load(model_src, corr, eprm) if isinstance(model_src, str) else \
            CorrectorModel(corr, eprm, like=model_src)
        return corr, model

    # reference trajectory (untimed): plain states at the curve points, and the teacher-forced
    # one-window error -- the proposal from the plain state U_w against 8 plain steps from U_w,
    # per case, so no error carries over from earlier windows
    ref = B.BatchedFVM(eparts, ecfg, device="cuda")
    ref.t_solver.update_cfl_dt(0.5)
    ref.t_solver.step(spinup)
    ref_window = ref.t_solver.graph_steps(8)
    tf_corr, tf_model = make_corr()
    tf_ro = CheckedRollout(tf_model, residual_ratio=gates[0][0], consistency=gates[0][1])
    tf_windows = min(args.windows, 50)
    tf_all, tf_ok = [], []
    ref_at = {}
    for w in range(1, args.windows + 1):
        if w <= tf_windows:
            tf_corr.cells.state = ref.cells.state
            tf_corr.t_solver._sync_prims()
            tf_ro._run_propose()
        ref_window()
        if w <= tf_windows:
            rel = case_rel(tf_ro.prop, ref.cells.state, ref)
            tf_all.append(rel)
            tf_ok.append(rel[tf_ro.ok])
        if w in curve_at:
            ref_at[w] = ref.cells.state.clone()
    tf_all, tf_ok = torch.cat(tf_all), torch.cat(tf_ok)
    fin = torch.isfinite(tf_all)
    teacher_forced = {
        "windows": tf_windows, "gate": {"residual_ratio": gates[0][0], "trapezoid_consistency": gates[0][1] or None},
        "rel_l2_all": {"mean": float(tf_all[fin].mean()), "max": float(tf_all[fin].max()),
                       "frac_below_1e-2": float((tf_all[fin] <= 1e-2).float().mean())},
        "rel_l2_accepted": ({"mean": float(tf_ok.mean()), "max": float(tf_ok.max()),
                             "frac_below_1e-2": float((tf_ok <= 1e-2).float().mean())} if tf_ok.numel() else None),
        "accept_rate": tf_ok.numel() / max(tf_all.numel(), 1)}
    del tf_corr, tf_model, tf_ro, ref, ref_window

    # control: the plain solver itself, its start state perturbed once by a seeded relative noise
    # of the corrector's mean one-window error -- how far the unsteady flow carries an error of
    # that size by itself over the same windows
    eps = teacher_forced["rel_l2_all"]["mean"]
    ctl = B.BatchedFVM(eparts, ecfg, device="cuda")
    ctl.t_solver.update_cfl_dt(0.5)
    ctl.t_solver.step(spinup)
    gen = torch.Generator(device="cuda").manual_seed(11)
    noise = torch.randn(ctl.cells.state.shape, generator=gen, device="cuda")
    ctl.cells.state = ctl.cells.state * (1.0 + eps * noise)
    ctl_window = ctl.t_solver.graph_steps(8)
    control = {"perturbation_rel": eps, "rel_l2_curve_by_window": {}}
    for w in range(1, (curve_at[-1] if curve_at else 0) + 1):
        ctl_window()
        if w in curve_at:
            rel = case_rel(ctl.cells.state, ref_at[w], ctl)
            ok = torch.isfinite(rel)
            control["rel_l2_curve_by_window"][str(w)] = {
                "mean": float(rel[ok].mean()) if bool(ok.any()) else None,
                "max": float(rel[ok].max()) if bool(ok.any()) else None}
    del ctl, ctl_window

    def rollout(ratio, consistency):
        corr, model = make_corr()
        ro = CheckedRollout(model, residual_ratio=ratio, consistency=consistency)
        # capture every CUDA graph before timing (capturing executes nothing; the state stays put)
        ro._run_propose()
        corr.t_solver._sync_prims()
        ro._fallback = corr.t_solver.graph_steps(8)
        f = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        f[0].record(stream)
        for _ in range(args.windows):
            ro.window()
        f[1].record(stream)
        torch.cuda.synchronize()
        ms_corr = f[0].elapsed_time(f[1])
        # the proposal + checks graph alone (it reads the state and writes only its own buffers)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(10):
            ro._run_propose()
        g1.record(stream)
        torch.cuda.synchronize()
        ms_propose = g0.elapsed_time(g1) / 10
        err, bad_plain, bad_corr = [], 0, 0
        for c in range(args.eval_cases):
            a = corr.case_state(c).double()
            r = plain.case_state(c).double()
            fa, fr = bool(torch.isfinite(a).all()), bool(torch.isfinite(r).all())
            bad_plain += not fr
            bad_corr += not fa
            if fa and fr:
                err.append(float(((a - r).norm() / r.norm()).item()))
        # drift curve (untimed second rollout from the same start): rel-L2 vs the plain trajectory
        corr2, model2 = make_corr()
        ro2 = CheckedRollout(model2, residual_ratio=ratio, consistency=consistency)
        curve = {}
        for w in range(1, (curve_at[-1] if curve_at else 0) + 1):
            ro2.window()
            if w in curve_at:
                rel = case_rel(corr2.cells.state, ref_at[w], corr2)
                ok = torch.isfinite(rel)
                curve[str(w)] = {"mean": float(rel[ok].mean()) if bool(ok.any()) else None,
                                 "max": float(rel[ok].max()) if bool(ok.any()) else None,
                                 "nonfinite_cases": int((~ok).sum())}
        del corr2, model2, ro2
        return {"residual_ratio": ratio, "trapezoid_consistency": consistency or None,
                "speedup": ms_plain / ms_corr, "ms_corrected": ms_corr,
                "rel_l2_curve_by_window": curve,
                "ms_per_window": {"corrected": ms_corr / args.windows, "plain": ms_plain / args.windows,
                                  "proposal_and_checks": ms_propose},
                "accept_rate": ro.accepted / max(ro.windows, 1),
                "windows_without_fallback": ro.full_windows / max(args.windows, 1),
                "rel_l2_vs_plain": {"max": max(err) if err else None, "mean": float(np.mean(err)) if err else None,
                                    "cases_compared": len(err)},
                "nonfinite_cases": {"plain": bad_plain, "corrected": bad_corr}}

    runs = [rollout(r, c) for r, c in gates]
    main, others = runs[0], runs[1:]
    return {"metric": "sim-time/s corrector+fallback over plain FVM", "value": main["speedup"], "unit": "x",
            "higher_is_better": True, "dtype": "bf16 GEMM / f32 state",
            "config": {"workload": "corrector_3d_sphere_k8" if three_d else "corrector_2d_k8",
                       "eval_cases": args.eval_cases, "eval_cells": int(plain.n_cells), "windows": args.windows,
                       "steps_per_rollout": 8 * args.windows, "spinup_steps": spinup,
                       "fvm": "SSP-RK3, fixed per-case dt (CFL 0.5)",
                       "net": "4 message-passing layers, width 64, SiLU, tcgen05 BF16 GEMMs",
                       "checks": f"drift <= 1e-4, residual norm <= {gates[0][0]}x, admissible state"
                                 + (f", trapezoid distance <= {gates[0][1]} k dt |r0|" if gates[0][1] else "")},
            "ms_plain": ms_plain, "teacher_forced_window_error": teacher_forced,
            "plain_perturbed_control": control,
            **{k: v for k, v in main.items() if k != "speedup"},
            "other_checks": others, "clocks": clk.summary()}


def corrector_bench(args, timed):
    """Learned k-step corrector (k = 8) + FVM fallback vs plain FVM on held-out cases: trains (or,
    with ``--checkpoint``, loads) the model, optionally saves it (``--save-checkpoint``), evaluates."""
    three_d = args.workload == "corrector3d"
    if args.train_cases is None:
        args.train_cases = 4 if three_d else 32
    if args.iters is None:
        args.iters = 2000 if three_d else 6000
    info = None
    if args.checkpoint:
        model_src = args.checkpoint
    else:
        model_src, info = corrector_train(args, three_d)
        if args.save_checkpoint:
            os.makedirs(os.path.dirname(os.path.abspath(args.save_checkpoint)), exist_ok=True)
            model_src.save(args.save_checkpoint, meta=info)
    out = corrector_evaluate(model_src, args, three_d)
    out.update({"n_gpus": 1, "data": "synthetic", "train": info,
                "model": args.checkpoint or "trained in this run"})
    print(json.dumps(out))


def corrector_bench_dp(args):
    """Data-parallel corrector training under torchrun (one rank per GPU, NCCL): every rank streams
    its share of the training cases and the gradients are averaged each iteration; rank 0 then
    saves the model (``--save-checkpoint``) and evaluates it alone, as ``corrector_bench`` does."""
    import torch.distributed as dist
    from datetime import timedelta
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    three_d = args.workload == "corrector3d"
    if args.iters is None:
        args.iters = 2000 if three_d else 6000
    model, info = corrector_train_streaming(args, three_d, group=dist.group.WORLD)
    dist.barrier()
    rank = dist.get_rank()
    dist.destroy_process_group()
    if rank != 0:
        return
    if args.save_checkpoint:
        os.makedirs(os.path.dirname(os.path.abspath(args.save_checkpoint)), exist_ok=True)
        model.save(args.save_checkpoint, meta=info)
    out = corrector_evaluate(model, args, three_d)
    out.update({"n_gpus": info["data_parallel_ranks"], "data": "synthetic", "train": info,
                "model": "trained in this run (data-parallel)"})
    print(json.dumps(out))


def ell_result(tables, reps: int = 20) -> dict:
    """The ELL operator seam (``SPMB200``, the drop-in for the reference's Triton ELL path) on the
    benchmark box's own operators, timed as the reference's micro-benchmark does
    (``benchmark/bench_utils.py:27-55``: random dense operand, warm-up, a loop of products) but with
    CUDA events: G_mats (LSQ gradients, [dim N] x [N + F_b], K = dim + 2) times the C-component
    state, flux_mat (divergence, [N] x [F], K = dim + 1) times C-component facet fluxes, and G_mats
    times one column (the reference script's case).  Algorithmic bytes per product: the ELL values
    and int32 columns (8 B per slot), the operand and the output once each (4 B per element).
    torch's CSR SpMM on the same matrices is timed beside it."""
    from fvm_solver_b200.sparse import SPMB200
    peak, peak_kind = measured_peaks()
    stream = torch.cuda.current_stream()
    C = tables.n_comp
    out = {}
    for name, A, B in (("G_mats_spmm", tables.ops.G_mats, C), ("flux_mat_spmm", tables.ops.flux_mat, C),
                       ("G_mats_spmv", tables.ops.G_mats, 1)):
        op = SPMB200(A, "cuda")
        X = torch.randn((A.shape[1], B), device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
        f = (lambda: op.spMM(X)) if B > 1 else (lambda: op.spMV(X[:, 0]))
        for _ in range(5):
            f()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            f()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        byts = op.M * op.K * 8 + A.shape[1] * B * 4 + op.M * B * 4
        Ad = A.to_sparse_csr().cuda()
        g = lambda: torch.sparse.mm(Ad, X)
        for _ in range(3):
            g()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            g()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_t = e0.elapsed_time(e1) / reps
        out[name] = {"rows": op.M, "K": op.K, "B": B, "ms": ms, "algorithmic_bytes": byts,
                     "achieved_gbs": byts / (ms / 1e3) / 1e9, "frac": byts / (ms / 1e3) / 1e9 / peak,
                     "torch_csr_ms": ms_t}
        del op, Ad
    torch.cuda.empty_cache()
    return {"peak_gbs": peak, "peak_source": peak_kind, "ops": out,
            "method": "CUDA events over 20 products after 5 warm-up ones (output allocated per call, "
                      "as SPM.spMM does)"}


def corrector_checkpoint_result(args, timed) -> dict:
    """The headline line's corrector key: the stored 2D model (trained offline by
    ``--workload corrector --save-checkpoint``) evaluated on the held-out cases; training is not
    part of this run."""
    if not os.path.exists(CORRECTOR_CKPT):
        return {"unavailable": "no stored corrector checkpoint"}
    d = torch.load(CORRECTOR_CKPT, map_location="cpu", weights_only=True)
    ev = argparse.Namespace(eval_cases=args.eval_cases, windows=args.windows)
    out = corrector_evaluate(CORRECTOR_CKPT, ev, three_d=False)
    out["model"] = {"checkpoint": os.path.relpath(CORRECTOR_CKPT, ROOT), "trained": d.get("meta", {})}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "taylor_green":
        return secondary(args)

    import torch.distributed as dist
    from fvm_solver_b200 import _lib, workloads as W
    from fvm_solver_b200.roofline import kernel_bytes, div_stage_bytes, step_compulsory_bytes, tableau_terms

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    if world > 1:
        torch.set_num_threads(max(1, (os.cpu_count() or 1) // world))   # ranks build their meshes at once
    case = W.taylor_green(n=args.n, seed=rank, device=f"cuda:{local}")
    eq = case.equation()
    sol = eq.t_solver
    N, F, Fb = eq.mesh.n_cells, eq.mesh.n_facets, eq.dev.n_bc
    lib = _lib.load()
    from fvm_solver_b200.autotune import autotune
    if args.launch:
        # fixed launch configuration (reproducing a profile of the benchmark's own kernels on a
        # smaller box): "cell=128,face=128,div_stage=64"; no prefetch, per-thread record loads
        from fvm_solver_b200 import autotune as AT
        AT.reset()
        tuned_full = {}
        for item in args.launch.split(","):
            k, _, bs = item.partition("=")
            AT.set_block_size(k, int(bs))
            tuned_full[k] = {"threads": int(bs), "prefetch": 0, "variant": "registers", "ms": {}}
    else:
        tuned_full = autotune(eq)
    tuned = {k: v["threads"] for k, v in tuned_full.items()}
    prefetch = {k: v["prefetch"] for k, v in tuned_full.items()}
    variants = {k: v["variant"] for k, v in tuned_full.items()}
    dv = tuned_full.get("div_stage", {})
    if "residual_ms" in dv:
        variants["residual"] = {"owner_computes" if dv["residual_variant"] else "separate": True,
                                "ms": {k: round(v, 5) for k, v in dv["residual_ms"].items()}}
    if os.environ.get("FVM_BENCH_VERBOSE"):
        for k, v in tuned_full.items():
            print(k, {c: round(ms * 1e3, 1) for c, ms in v["ms"].items()}, file=sys.stderr)

    # warm-up
    sol.step(args.warmup)
    torch.cuda.synchronize()

    # timed region 1: K steps replayed from one CUDA graph
    replay = sol.graph_steps(args.steps)
    replay()                                 # untimed warm-up replay (the first one uploads the graph)
    barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        replay()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)

        # timed region 2: K eager steps with every launch bracketed by CUDA events
        cap = args.steps * 64 + 64
        _lib.check(lib.fvm_profile_start(cap), "fvm_profile_start")
        sol.step(args.steps)
        n_launch = lib.fvm_profile_stop()
        torch.cuda.synchronize()
    if n_launch < 0:
        raise RuntimeError("profiling buffer overflow")
    ids = np.zeros(n_launch, np.int32)
    kms = np.zeros(n_launch, np.float32)
    got = lib.fvm_profile_read(n_launch, ids.ctypes.data, kms.ctypes.data)
    if got != n_launch:
        raise RuntimeError("fvm_profile_read failed")
    clocks = clk.summary()

    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells_total = N * world
    value = cells_total * args.steps / (ms_max / 1e3)

    # per-kernel accounting (timed region 2)
    kern = {}
    for kid in np.unique(ids):
        sel = ids == kid
        kern[_lib.KERNEL_NAMES[int(kid)]] = {"launches": int(sel.sum()), "ms_total": float(kms[sel].sum()),
                                              "ms_mean": float(kms[sel].mean())}
    tot = sum(v["ms_total"] for v in kern.values())
    for v in kern.values():
        v["share"] = v["ms_total"] / tot
    def launch_bytes(widths):
        kb = kernel_bytes(3, N, F, Fb, eq.dev.kf, widths=widths)
        out = {"cell": kb["cell"], "face": kb["face"], "bc": kb["bc"]}
        out["div_stage"] = float(np.mean(div_stage_bytes(3, N, F, Fb, tableau_terms(sol.tab), eq.dev.kf, widths)))
        return out
    per_launch = launch_bytes("element")             # 4 B per used element (the roofline's count)
    per_launch_stored = launch_bytes("stored")       # 4 B per stored float, row padding included
    dom = max((k for k in kern if k in per_launch), key=lambda k: kern[k]["ms_total"])
    peak, peak_kind = measured_peaks()
    achieved = per_launch[dom] / (kern[dom]["ms_mean"] / 1e3) / 1e9
    achieved_stored = per_launch_stored[dom] / (kern[dom]["ms_mean"] / 1e3) / 1e9
    step_bytes = step_compulsory_bytes(3, N, F, sol.tab.stages)
    step_gbs = step_bytes / (ms_max / args.steps / 1e3) / 1e9
    traffic = traffic_src = None
    tf = os.path.join(ROOT, "profiles", "dram_bytes_per_cell.json")
    if os.path.exists(tf):
        d = json.load(open(tf))
        if dom in d.get("kernels", {}):
            traffic = d["kernels"][dom] * N
            traffic_src = d.get("source")
    for k, v in kern.items():
        if k in per_launch:
            v["algorithmic_bytes_per_launch"] = per_launch[k]
            v["achieved_gbs"] = per_launch[k] / (v["ms_mean"] / 1e3) / 1e9
            v["frac"] = v["achieved_gbs"] / peak
            v["stored_bytes_per_launch"] = per_launch_stored[k]

    # end-to-end through the public API with host buffers
    ke = args.e2e_steps or max(args.steps, 50)
    ring = 4                                          # distinct host states, cycled
    host_in = [torch.empty((N, 5), dtype=torch.float32).pin_memory() for _ in range(ring)]
    host_out = [torch.empty((N, 5), dtype=torch.float32).pin_memory() for _ in range(ring)]
    for h in host_in:
        sol.step(1)
        h.copy_(eq.cells.state.cpu())
    sol.step_host(host_in[:2], host_out[:2])          # untimed: creates the copy streams, slots and graphs
    torch.cuda.synchronize()

    def e2e_time(run) -> float:
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        run()
        f1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([f0.elapsed_time(f1)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return cells_total * ke / (float(t.item()) / 1e3)

    # (a) streamed: ke independent host states, each copied in, stepped once and copied out;
    #     the copies of the neighbouring states overlap each step
    e2e_value = e2e_time(lambda: sol.step_host([host_in[i % ring] for i in range(ke)],
                                               [host_out[i % ring] for i in range(ke)]))

    # (b) chained: the state goes through the host every step (each step's input is the previous
    #     step's output read back), so nothing can overlap
    def chained():
        a, b = host_in[0], host_out[0]
        for _ in range(ke):
            eq.cells.copy_from(a, non_blocking=True)      # H2D (pinned), stream-ordered after the last D2H
            sol.step(1)
            b.copy_(eq.cells.state, non_blocking=True)    # D2H of the step's result
            a, b = b, a
    e2e_chained = e2e_time(chained)

    # the transfer bound of (a): one state in and one state out at once, on two copy streams
    # (what every streamed step has to move), timed alone
    def copy_ms(h2d: bool, d2h: bool, reps: int = 5) -> float:
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        dev_in, dev_out = torch.empty((N, 5), device="cuda"), eq.cells.state.clone()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
        for _ in range(reps):
            if h2d:
                with torch.cuda.stream(s_in):
                    dev_in.copy_(host_in[1], non_blocking=True)
            if d2h:
                with torch.cuda.stream(s_out):
                    host_out[1].copy_(dev_out, non_blocking=True)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        g1.record(stream)
        torch.cuda.synchronize()
        return g0.elapsed_time(g1) / reps
    copy_pair, copy_h2d, copy_d2h = copy_ms(True, True), copy_ms(True, False), copy_ms(False, True)

    # the device bound of (a): one state's device work (copy into the state, restart, one step,
    # copy out -- the graph step_host replays per state), replayed back to back without copies
    per_state = sol._host_stage(1)["graphs"][0]
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(10):
        per_state.replay()
    g1.record(stream)
    torch.cuda.synchronize()
    state_ms = g0.elapsed_time(g1) / 10
    e2e_step_ms = cells_total * 1e3 / e2e_value
    e2e_bound_ms = max(copy_pair, state_ms)

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.sample_n)                 # on the host cores, at N = 1 only
    if rank == 0 and not args.no_cpu_baseline:
        parity = parity_check(args.sample_n)
    launches_per_step = n_launch / args.steps
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        # The north star's other targets, each with its own CUDA-event timing and clock record:
        # config 1 (2D channel, with its trajectory against the oracle), config 3 (batched
        # ensemble vs the cases one by one) and configs 4 (corrector from a stored checkpoint).
        timed = graph_timer(stream)
        extras["channel_cylinder"] = channel_cylinder_result(50, 5, args.drift_steps, not args.no_cpu_baseline, timed)
        extras["ensemble"] = ensemble_result(args.cases, 20, 5, timed, cfl=args.ensemble_cfl or ENSEMBLE_CFL)
        extras["corrector"] = corrector_checkpoint_result(args, timed)
        extras["ell"] = ell_result(eq.tables)
    if rank == 0:
        out = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "taylor_green_periodic_box_rk4_cfl0.5", "points_per_axis": args.n,
                       "cells_per_gpu": N, "facets_per_gpu": F, "state": "fp32 [N,5]",
                       "l2": "inputs larger than L2 (>1 GB touched per stage), no flush",
                       "parallelism": f"{world} independent boxes (one per rank)", "timing": "cuda graph replay",
                       "block_sizes": tuned, "l2_prefetch": prefetch, "kernel_variants": variants},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "traffic_source": traffic_src,
                         "algorithmic_bytes_per_launch": per_launch[dom],
                         "bytes": "4 B per used element (row padding not counted)",
                         "frac_stored": achieved_stored / peak,
                         "stored_bytes_per_launch": per_launch_stored[dom],
                         "step_compulsory_bytes": step_bytes,
                         "step_compulsory_gbs": step_gbs,
                         "step_compulsory_frac": step_gbs / peak,
                         "step_compulsory_def": "one-pass stage traffic x stages: 4 B x (per cell 2C + dim KG + KG "
                                                "+ K + K dim + 2 + 4K; per facet 2 dim + 3); 328 B per cell-stage "
                                                "in 3D"},
            "kernels": kern,
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": N * 5 * 4,
                    "d2h_bytes_per_step": N * 5 * 4, "steps": ke,
                    "mode": "TSolver.step_host: independent pinned host states, each copied in, stepped "
                            "once (RK4, CFL dt from the state; one CUDA-graph replay) and copied out; "
                            "copies on two streams overlap the neighbouring steps",
                    "chained_value": e2e_chained,
                    "bound": {"kind": "pcie" if copy_pair > state_ms else "device",
                              "ms_per_step": e2e_step_ms, "copy_in_and_out_ms": copy_pair,
                              "copy_in_ms": copy_h2d, "copy_out_ms": copy_d2h,
                              "device_state_ms": state_ms, "device_step_ms": ms_max / args.steps,
                              "frac": e2e_bound_ms / e2e_step_ms},
                    "chained_mode": "state round-trips through the host every step (no overlap possible)"},
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "clocks": clocks,
            **extras,
        }
        print(json.dumps(out))
    del replay
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
