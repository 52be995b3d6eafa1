"""Batched ensemble: many independent meshes of uneven size advanced by the same launches.

The cases' kernel tables are concatenated (cells, facets, boundary facets and characteristic
facets each contiguous per case; every index made global) and tagged with per-case arrays
(``cell_case``, ``face_case``, ``bc_case``, ``ch_off``, transport coefficients).  One launch of
each residual kernel then covers every case, so a 2 000-cell case no longer pays a whole
GPU-underfilling launch sequence of its own; per-case quantities (time step, characteristic-BC
sound-speed mean, CFL and conservation reductions) stay per case inside the kernels.  Results
are bitwise identical to running each case alone (``tests/test_gpu_batched.py``).

``BatchedFVM`` exposes the attributes the solvers of ``solvers.py`` use, so ``AB3`` (the
ensemble's integrator: Adams-Bashforth 3 after two SSP-RK3 start-up steps, fixed per-case dt from
the initial CFL condition) and the ``Butcher`` family run on it unchanged, including CUDA-graph
capture of whole steps.
"""
from __future__ import annotations

import concurrent.futures as cfut
import multiprocessing as mp
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .equation import FVMCells, FluidConstitution2D, FluidConstitution3D
from .tables import KernelTables


@dataclass
class CaseTables:
    """Host tables of one case (picklable, built in a worker process)."""
    kt: KernelTables
    state0: torch.Tensor
    mu: float
    mu_b: float
    kappa: float
    name: str
    gas: tuple          # (T_0, S_const, C_v, gamma, v_factor, lim_p)


def build_case_tables(case) -> CaseTables:
    cfg = case.cfg
    T = case.tables()
    return CaseTables(T.kernel, case.state0, float(cfg.viscosity), float(cfg.visc_bulk), float(cfg.thermal_cond),
                      case.name, (cfg.T_0, cfg.S_const, cfg.C_v, cfg.gamma, cfg.v_factor, cfg.lim_p))


def _ensemble_worker(args):
    from .workloads import ensemble_case, sphere_case
    i, base_seed, family, cells = args
    if family == "sphere":
        return build_case_tables(sphere_case(i, device="cpu", base_seed=base_seed, cells=cells))
    return build_case_tables(ensemble_case(i, device="cpu", base_seed=base_seed))


def _worker_init():
    # one intra-op thread per worker process: the workers already run in parallel
    torch.set_num_threads(1)


def _table_worker_loop(jobs, results):
    _worker_init()
    while True:
        item = jobs.get()
        if item is None:
            return
        jid, job = item
        results.put((jid, _ensemble_worker(job)))


class TableWorkers:
    """Spawned host processes that build case tables for a long stream of jobs (corrector
    training).  Each worker takes (id, job) items from one queue and puts (id, tables) on another.
    A worker that dies (whatever the cause) is replaced and every job that has not come back is
    queued again; a result that arrives twice is kept once.  ``restarts`` counts replaced workers,
    ``exit_codes`` their exit codes."""

    def __init__(self, workers: int):
        self.ctx = mp.get_context("spawn")
        self.jobs, self.results = self.ctx.Queue(), self.ctx.Queue()
        self.procs = [self._start() for _ in range(max(1, workers))]
        self.pending: dict = {}           # id -> job, submitted and not yet returned
        self.done: dict = {}              # id -> tables, returned and not yet taken
        self.taken: set = set()
        self.restarts, self.exit_codes = 0, []

    def _start(self):
        p = self.ctx.Process(target=_table_worker_loop, args=(self.jobs, self.results), daemon=True)
        p.start()
        return p

    def submit(self, jid, job):
        self.pending[jid] = job
        self.jobs.put((jid, job))

    def _replace_dead(self):
        dead = [i for i, p in enumerate(self.procs) if not p.is_alive()]
        if not dead:
            return
        for i in dead:
            self.exit_codes.append(self.procs[i].exitcode)
            self.procs[i] = self._start()
        self.restarts += len(dead)
        for jid, job in self.pending.items():          # whichever job a dead worker held
            self.jobs.put((jid, job))

    def get(self, jid, timeout: float = 3600.0):
        import queue
        import time
        t0 = time.time()
        while jid not in self.done:
            if time.time() - t0 > timeout:
                raise TimeoutError(f"table job {jid} did not come back in {timeout:.0f} s")
            self._replace_dead()
            try:
                rid, res = self.results.get(timeout=5.0)
            except queue.Empty:
                continue
            if rid in self.taken or rid in self.done:
                continue                                 # a resubmitted job's second result
            self.pending.pop(rid, None)
            self.done[rid] = res
        self.taken.add(jid)
        return self.done.pop(jid)

    def close(self):
        for _ in self.procs:
            self.jobs.put(None)
        for p in self.procs:
            p.join(timeout=10)
            if p.is_alive():
                p.terminate()


def build_ensemble_tables(n_cases: int, base_seed: int = 1234, workers: int = 0, family: str = "channel",
                          cells=(300_000, 800_000), indices=None) -> list:
    """Per-case tables of a seeded ensemble -- ``family`` "channel" (2D channel-cylinder cases) or
    "sphere" (3D flow over a sphere, ``cells`` the tet-count range); ``workers > 0`` builds them in
    spawned processes.  ``indices`` builds only those cases of the ensemble (one rank's share)."""
    ids = range(n_cases) if indices is None else list(indices)
    jobs = [(i, base_seed, family, tuple(cells)) for i in ids]
    if not jobs:
        return []
    if workers > 0:
        ctx = mp.get_context("spawn")
        with cfut.ProcessPoolExecutor(max_workers=workers, mp_context=ctx, initializer=_worker_init) as ex:
            return list(ex.map(_ensemble_worker, jobs, chunksize=4))
    return [_ensemble_worker(j) for j in jobs]


def concat_tables(parts: list) -> tuple:
    """Concatenate per-case KernelTables into one batched table set + per-case arrays."""
    kts = [p.kt for p in parts]
    dim, C = kts[0].dim, kts[0].n_comp
    kg, kf = kts[0].kg, kts[0].kf
    for k in kts:
        if (k.dim, k.kg, k.kf) != (dim, kg, kf):
            raise ValueError("batched cases must share dim and stencil widths")
    Ns = np.array([k.n_cells for k in kts])
    Fs = np.array([k.n_facets for k in kts])
    Bs = np.array([k.n_bc for k in kts])
    Hs = np.array([k.n_char for k in kts])
    co, fo, bo, ho = (np.concatenate([[0], np.cumsum(x)[:-1]]) for x in (Ns, Fs, Bs, Hs))
    Nt, Ft, Bt, Ht = int(Ns.sum()), int(Fs.sum()), int(Bs.sum()), int(Hs.sum())
    i32 = torch.int32

    def cat(name, axis, off=None, neg_keep=False):
        out = []
        for c, k in enumerate(kts):
            a = getattr(k, name)
            if off is not None:
                a = a.long()
                if neg_keep:
                    a = torch.where(a >= 0, a + int(off[c]), a)
                else:
                    a = a + int(off[c])
                a = a.to(i32)
            out.append(a)
        return torch.cat(out, dim=axis).contiguous()

    gcols = []
    for c, k in enumerate(kts):
        g = k.g_cols.long()
        g = torch.where(g < k.n_cells, g + int(co[c]), g - k.n_cells + Nt + int(bo[c]))
        gcols.append(g.to(i32))
    kt = KernelTables(
        dim=dim, n_comp=C, n_cells=Nt, n_facets=Ft, n_bc=Bt, n_char=Ht, kg=kg, kf=kf,
        g_vals=cat("g_vals", 2), g_cols=torch.cat(gcols, 1).contiguous(), nb_slot=cat("nb_slot", 0),
        disp=cat("disp", 2), eps=cat("eps", 0), c2f=cat("c2f", 1, fo), side=cat("side", 0),
        f_vals=cat("f_vals", 1), f_cols=cat("f_cols", 1, fo), inv_h=cat("inv_h", 0), volumes=cat("volumes", 0),
        centroids=cat("centroids", 0),
        fcell=cat("fcell", 0, co), fbc=cat("fbc", 0, bo, True), normals=cat("normals", 0), fsize=cat("fsize", 0),
        xorth=cat("xorth", 0), inv_d=cat("inv_d", 0),
        bc_face=cat("bc_face", 0, fo), bc_side=cat("bc_side", 0), bc_cell=cat("bc_cell", 0, co),
        bc_kind=cat("bc_kind", 0), bc_b=cat("bc_b", 0), bc_l=cat("bc_l", 0), bc_ga=cat("bc_ga", 0),
        bc_gb=cat("bc_gb", 0), bc_char=cat("bc_char", 0, ho, True), ch_cell=cat("ch_cell", 0, co),
        ch_normal=cat("ch_normal", 0), ch_rho=cat("ch_rho", 0), ch_vn=cat("ch_vn", 0), ch_vt=cat("ch_vt", 0),
        ch_p=cat("ch_p", 0))
    case_arrays = dict(
        cell_case=torch.repeat_interleave(torch.arange(len(kts), dtype=i32), torch.from_numpy(Ns)),
        face_case=torch.repeat_interleave(torch.arange(len(kts), dtype=i32), torch.from_numpy(Fs)),
        bc_case=torch.repeat_interleave(torch.arange(len(kts), dtype=i32), torch.from_numpy(Bs)),
        ch_off=torch.from_numpy(np.concatenate([[0], np.cumsum(Hs)]).astype(np.int32)),
        case_mu=torch.tensor([p.mu for p in parts], dtype=torch.float32),
        case_mu_b=torch.tensor([p.mu_b for p in parts], dtype=torch.float32),
        case_kappa=torch.tensor([p.kappa for p in parts], dtype=torch.float32))
    offsets = dict(cells=np.concatenate([co, [Nt]]), facets=np.concatenate([fo, [Ft]]))
    return kt, case_arrays, offsets


class _BatchMeshInfo:
    def __init__(self, n_cells, dim):
        self.n_cells = n_cells
        self.dim = dim


class BatchedDeviceMesh:
    def __init__(self, kt: KernelTables, case_arrays: dict, device):
        from .equation import DeviceMesh
        self.base = DeviceMesh(kt, device)
        self.t = self.base.t
        self.device = self.base.device
        self.n_comp, self.n_cells, self.n_facets, self.n_bc = kt.n_comp, kt.n_cells, kt.n_facets, kt.n_bc
        self.dim, self.row, self.grow, self.kf = kt.dim, self.base.row, self.base.grow, kt.kf
        self.case = {k: v.contiguous().to(self.device) for k, v in case_arrays.items()}
        m = self.base.struct
        m.n_cases = int(case_arrays["case_mu"].numel())
        for k, v in self.case.items():
            setattr(m, k, _lib.ptr(v))
        self.struct = m


class BatchedFVM:
    """Several independent meshes stepped together (see module docstring)."""

    def __init__(self, parts: list, cfg, device="cuda"):
        self.lib = _lib.load()
        self.device = torch.device(device)
        self.parts = parts
        self.n_cases = len(parts)
        gas = {p.gas for p in parts}
        if len(gas) != 1:
            raise ValueError("batched cases must share T_0, S_const, C_v, gamma, v_factor and lim_p")
        kt, ca, off = concat_tables(parts)
        self.kt = kt
        self.offsets = off
        self.dev = BatchedDeviceMesh(kt, ca, self.device)
        T_0, S, C_v, gamma, v_factor, lim_p = next(iter(gas))
        self.phys = _lib.Physics(T_0=T_0, mu=parts[0].mu, mu_b=parts[0].mu_b, S_const=S, C_v=C_v, gamma=gamma,
                                 kappa=parts[0].kappa, v_factor=v_factor, lim_p=lim_p)
        self.n_comp = C = kt.n_comp
        self.mesh = _BatchMeshInfo(kt.n_cells, kt.dim)
        from .equation import Work
        self.work = Work(self.dev)
        self.work.red = torch.zeros(_lib.FVM_RED_DOUBLES + 8 * self.n_cases, dtype=torch.float64, device=self.device)
        self.work.struct.red = _lib.ptr(self.work.red)
        self.grads = torch.zeros((kt.n_cells, self.dev.grow), device=self.device)
        self.has_grads = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._has_grads_host = False
        phy = (FluidConstitution2D if kt.dim == 2 else FluidConstitution3D)(cfg)
        self.cells = FVMCells(kt.n_cells, C, phy, init_val=torch.cat([p.state0 for p in parts]), device=self.device)
        from .solvers import get_solver
        self.t_solver = get_solver(self.cells, self, cfg)

        self.active = torch.ones(self.n_cases, dtype=torch.uint8, device=self.device)

    def use_case_mask(self, on: bool = True):
        """Let ``self.active`` (device bytes, one per case) freeze cases: every kernel launched for
        this batch afterwards -- also from CUDA graphs captured afterwards, which read the mask at
        replay -- skips the cases whose byte is 0."""
        self.dev.struct.case_active = _lib.ptr(self.active) if on else None

    def case_slice(self, c: int) -> slice:
        return slice(int(self.offsets["cells"][c]), int(self.offsets["cells"][c + 1]))

    def case_state(self, c: int) -> torch.Tensor:
        return self.cells.state[self.case_slice(c)]

    @property
    def n_cells(self) -> int:
        return self.mesh.n_cells
