"""Time integrators on the device (mirrors ``time_fvm/time_solvers/integrators.py`` / ``t_solvers.py``).

Every solver advances ``FVMCells.state`` with ``fvm_step`` / ``fvm_multistep``: the stage
combinations, the conserved -> primitive conversion and the step-size update all run inside the
stage kernels; ``dt`` lives on the device, so a step issues no host synchronisation and whole
steps can be captured in a CUDA graph (``TSolver.graph_steps``).

* ``Butcher(name)``       -- fixed (or CFL) dt, tableau ``name`` (``integrators.py:349-393``)
* ``ButcherAdapt(name)``  -- embedded error estimate + ``Adaptive.update_stepsize``
                             (``integrators.py:42-62, 305-346``)
* ``RK3_SSP4``            -- the hand-unrolled four-stage SSP-RK3 (``integrators.py:65-94``): the
                             same tableau as ``Butcher_Tables("RK3_SSP4")`` with the low-order
                             estimate ``U_b - U_0 = (k1 + k2) / 2``
* ``AB3``                 -- Adams-Bashforth 3 after two SSP-RK3 start-up steps (restated; the
                             reference's ``Adams3PC`` cannot run, ``integrators.py:111``)
* ``SSP_RK3``             -- three-stage Shu-Osher SSP-RK3 tableau (restated from
                             ``integrators_bad.py:13-35``)

``cfg.cfl`` (when set) recomputes dt = cfl * min h / (|u| + c) in FP64 after every step.
"""
from __future__ import annotations

import ctypes as ct

import torch

from . import _lib

_T = {
    # integrators.py:216-226
    "RK4": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1.0, 0]],
            [1 / 6, 1 / 3, 1 / 3, 1 / 6], [1 / 4] * 4),
    # integrators.py:228-238
    "RK3_SSP4": ([[0, 0, 0, 0], [0.5, 0, 0, 0], [0.5, 0.5, 0, 0], [1 / 6, 1 / 6, 1 / 6, 0]],
                 [1 / 6, 1 / 6, 1 / 6, 1 / 2], [1 / 4] * 4),
    # integrators.py:240-251
    "RK3_SSP5": ([[0, 0, 0, 0, 0],
                  [0.37726891511710, 0, 0, 0, 0],
                  [0.37726891511710, 0.37726891511710, 0, 0, 0],
                  [0.16352294089771, 0.16352294089771, 0.16352294089771, 0, 0],
                  [0.14904059394856, 0.14831273384724, 0.14831273384724, 0.34217696850008, 0]],
                 [0.19707596384481, 0.11780316509765, 0.11709725193772, 0.27015874934251, 0.29786487010104],
                 [1 / 5] * 5),
    # integrators.py:253-265
    "RK3_SSP6": ([[0, 0, 0, 0, 0, 0],
                  [0.28422, 0, 0, 0, 0, 0],
                  [0.28422, 0.28422, 0, 0, 0, 0],
                  [0.23071, 0.23071, 0.23071, 0, 0, 0],
                  [0.13416, 0.13416, 0.13416, 0.16528, 0, 0],
                  [0.13416, 0.13416, 0.13416, 0.16528, 0.28422, 0]],
                 [0.17016, 0.17016, 0.10198, 0.12563, 0.21604, 0.21604], [1 / 6] * 6),
    # integrators.py:267-278
    "RK4_SSP5": ([[0, 0, 0, 0, 0],
                  [0.39175222700392, 0, 0, 0, 0],
                  [0.21766909633821, 0.36841059262959, 0, 0, 0],
                  [0.08269208670950, 0.13995850206999, 0.25189177424738, 0, 0],
                  [0.06796628370320, 0.11503469844438, 0.20703489864929, 0.54497475021237, 0]],
                 [0.14681187618661, 0.24848290924556, 0.10425883036650, 0.27443890091960, 0.22600748319395],
                 [1 / 5] * 5),
    # integrators.py:280-296
    "RK4_SSP10": ([[0] * 10,
                   [1 / 6] + [0] * 9,
                   [1 / 6] * 2 + [0] * 8,
                   [1 / 6] * 3 + [0] * 7,
                   [1 / 6] * 4 + [0] * 6,
                   [1 / 15] * 5 + [0] * 5,
                   [1 / 15] * 5 + [1 / 6] + [0] * 4,
                   [1 / 15] * 5 + [1 / 6] * 2 + [0] * 3,
                   [1 / 15] * 5 + [1 / 6] * 3 + [0] * 2,
                   [1 / 15] * 5 + [1 / 6] * 4 + [0]],
                  [1 / 10] * 10, [1 / 5, 0, 0, 3 / 10, 0, 0, 1 / 5, 0, 3 / 10, 0]),
    # three-stage Shu-Osher SSP-RK3
    "SSP_RK3": ([[0, 0, 0], [1, 0, 0], [0.25, 0.25, 0]], [1 / 6, 1 / 6, 2 / 3], [0.5, 0.5, 0]),
}


def tableau_names():
    return sorted(_T)


def make_tableau(name: str, adaptive=False, cfl: float | None = None, b2=None, atol=2e-3, rtol=2e-3,
                 mtol=1e-6, alphas=(0.8, 0.995), order=4) -> _lib.Tableau:
    if name not in _T:
        raise NotImplementedError("Unknown Butcher tableau")
    A, b, b2d = _T[name]
    b2 = b2d if b2 is None else b2
    t = _lib.Tableau()
    t.stages = len(b)
    for i, row in enumerate(A):
        for j, v in enumerate(row):
            t.a[i][j] = float(torch.tensor(v, dtype=torch.float32))
    for j in range(len(b)):
        t.b[j] = float(torch.tensor(b[j], dtype=torch.float32))
        t.b2[j] = float(torch.tensor(b2[j], dtype=torch.float32))
    t.adaptive = int(adaptive)
    t.atol, t.rtol, t.mtol = atol, rtol, mtol
    t.alpha_hi_err, t.alpha_lo_err = alphas
    t.order = order
    t.cfl = float(cfl) if cfl else 0.0
    return t


class TSolver:
    """Device time stepper for one ``FVMEquation``."""

    n_k = 0

    def __init__(self, cells, eq, cfg):
        self.cfg = cfg
        self.cells = cells
        self.eq = eq
        self.lib = eq.lib
        dev = eq.device
        self.n_steps = cfg.n_iter
        self.end_t = cfg.end_t
        self.print_i = cfg.print_i
        N, C = eq.mesh.n_cells, eq.n_comp
        self.prims = torch.zeros((N, eq.dev.row), device=dev)
        self.k = torch.zeros((max(self.n_k, 1), N, C), device=dev)
        self.n_cases = max(1, int(getattr(eq, "n_cases", 0) or 0))
        self.dt = torch.full((self.n_cases,), cfg.dt if cfg.dt is not None else 0.0, dtype=torch.float32,
                             device=dev)
        self.cons = None
        self._prims_version = -1
        self.t = 0.0
        self.steps_done = 0
        self.bufs = _lib.SolverBufs(state=_lib.ptr(cells.state), prims=_lib.ptr(self.prims),
                                    grads=_lib.ptr(eq.grads), k=_lib.ptr(self.k), dt=_lib.ptr(self.dt),
                                    has_grads=_lib.ptr(eq.has_grads), cons=None)
        self.cfl = getattr(cfg, "cfl", None)      # a reference ConfigFVM has no cfl field
        if self.cfl:
            self.update_cfl_dt()

    # -- helpers ------------------------------------------------------------------------------
    fused = False     # True: whole steps as one cooperative launch (fvm_step_fused); see autotune

    def _step_fn(self):
        return self.lib.fvm_step_fused if self.fused else self.lib.fvm_step

    def fused_status(self) -> int:
        """1 if a grid-barrier wait of a fused step ever gave up (results invalid), else 0."""
        out = ct.c_int32(0)
        _lib.check(self.lib.fvm_fused_status(ct.byref(self.eq.work.struct), ct.byref(out)), "fvm_fused_status")
        return int(out.value)

    def track_conservation(self, on: bool = True):
        """Record the FP64 totals sum vol * U after every step in ``self.cons`` (device)."""
        if on and self.cons is None:
            self.cons = torch.zeros((self.n_cases, self.eq.n_comp), dtype=torch.float64, device=self.eq.device)
        self.bufs.cons = _lib.ptr(self.cons) if on else None

    def update_cfl_dt(self, cfl: float | None = None):
        cfl = cfl or self.cfl
        _lib.check(self.lib.fvm_cfl_dt(ct.byref(self.eq.dev.struct), ct.byref(self.eq.phys),
                                       _lib.ptr(self.cells.state), float(cfl), _lib.ptr(self.dt),
                                       ct.byref(self.eq.work.struct), _lib.stream_ptr()), "fvm_cfl_dt")

    def _state_to_prims(self):
        _lib.check(self.lib.fvm_state_to_prims(ct.byref(self.eq.dev.struct), ct.byref(self.eq.phys),
                                               _lib.ptr(self.cells.state), _lib.ptr(self.prims),
                                               _lib.stream_ptr()), "fvm_state_to_prims")

    def _sync_prims(self):
        if self._prims_version != self.cells.version:
            self._state_to_prims()
            self._prims_version = self.cells.version

    def _step(self):
        raise NotImplementedError

    def _solve_step(self, t=None):
        self._sync_prims()
        self._step()
        self.eq._has_grads_host = True
        self.steps_done += 1

    def step(self, n: int = 1):
        for _ in range(n):
            self._solve_step()

    def graph_steps(self, n: int):
        """Capture ``n`` steps in a CUDA graph; returns a callable that replays them."""
        self._sync_prims()
        s = torch.cuda.Stream(device=self.eq.device)
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            # the capture must not start with an un-synced conversion
            with torch.cuda.graph(g, stream=s):
                for _ in range(n):
                    self._step()
        torch.cuda.current_stream().wait_stream(s)

        def replay():
            g.replay()
            self.eq._has_grads_host = True
            self.steps_done += n

        replay.graph = g
        return replay

    # -- host-resident states ------------------------------------------------------------------
    def _restart(self, dt0: torch.Tensor):
        """Make the next step behave as on a freshly built solver holding the current state: no
        carried limiter gradients, no multistep history, the time step of ``dt0`` (or, with a CFL
        number, recomputed from the state as the constructor does)."""
        self.eq.has_grads.zero_()
        self.eq._has_grads_host = False
        self.dt.copy_(dt0)
        if hasattr(self, "n_hist"):
            self.n_hist, self.head = 0, 0
        if self.cfl:
            self.update_cfl_dt()

    def _host_stage(self, steps: int) -> dict:
        """Device slots, copy streams and the per-slot CUDA graphs of ``step_host``.  The graph of
        slot s copies slot s into the state, restarts the solver (``_restart``), converts the
        state to primitives, takes ``steps`` steps and copies the result to output slot s.  The
        graphs are kept for the next call with the same ``steps``, step form, CFL number and
        conservation tracking (all baked into the captured launches); block sizes set later by
        the autotuner do not reach them (results do not depend on block sizes)."""
        dev = self.eq.device
        N, C = self.cells.state.shape
        st = getattr(self, "_host_st", None)
        if st is None:
            st = self._host_st = {
                "h2d": torch.cuda.Stream(device=dev), "d2h": torch.cuda.Stream(device=dev),
                "slot_in": [torch.empty((N, C), device=dev) for _ in range(2)],
                "slot_out": [torch.empty((N, C), device=dev) for _ in range(2)],
                "dt0": torch.empty_like(self.dt), "key": None}
        key = (steps, self.fused, self.cfl, self.bufs.cons)
        if st["key"] != key:
            st["graphs"] = None
            s = torch.cuda.Stream(device=dev)
            s.wait_stream(torch.cuda.current_stream(dev))
            graphs = []
            for slot in range(2):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.stream(s):
                    with torch.cuda.graph(g, stream=s):
                        self.cells.state.copy_(st["slot_in"][slot])
                        self._restart(st["dt0"])
                        self._state_to_prims()
                        for _ in range(steps):
                            self._step()
                        st["slot_out"][slot].copy_(self.cells.state)
                graphs.append(g)
            torch.cuda.current_stream(dev).wait_stream(s)
            # host-side multistep counters after the captured steps (set after every replay)
            st["hist"] = (self.n_hist, self.head) if hasattr(self, "n_hist") else None
            st["graphs"], st["key"] = graphs, key
        return st

    def step_host(self, inputs, outputs, steps: int = 1):
        """Advance a stream of independent host states: ``outputs[i]`` <- ``inputs[i]`` after
        ``steps`` steps, each state started afresh (see ``_restart``; the time step in force at
        the call is every state's initial one).

        ``inputs`` and ``outputs`` are sequences of contiguous float32 [N, C] host tensors, pinned
        for the copies to run asynchronously (an output may appear twice; the later state wins;
        an output must not also be an input, since the two copy streams are not ordered).
        Each state's device work is one CUDA-graph replay on the current stream, through two
        device slots each way; the copies run on two copy streams, so the host->device copy of
        state i+1 and the device->host copy of state i-1 overlap the steps of state i, and the
        host does not wait.  The call returns once everything is queued: synchronise the current
        stream before reading ``outputs``.  The solver is left holding the last state's result.
        """
        n = len(inputs)
        if len(outputs) != n:
            raise ValueError("step_host needs as many outputs as inputs")
        if n == 0:
            return outputs
        N, C = self.cells.state.shape
        for t in (*inputs, *outputs):
            if t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous() or tuple(t.shape) != (N, C):
                raise ValueError(f"step_host needs contiguous float32 host tensors of shape [{N}, {C}]")
        if {t.data_ptr() for t in inputs} & {t.data_ptr() for t in outputs}:
            raise ValueError("step_host: an output buffer is also an input")
        dev = self.eq.device
        comp = torch.cuda.current_stream(dev)
        st = self._host_stage(steps)
        h2d, d2h, slot_in, slot_out, graphs = st["h2d"], st["d2h"], st["slot_in"], st["slot_out"], st["graphs"]
        in_ready = [torch.cuda.Event() for _ in range(2)]
        slot_free = [torch.cuda.Event() for _ in range(2)]      # graph of the slot's last state done
        out_free = [torch.cuda.Event() for _ in range(2)]
        st["dt0"].copy_(self.dt)
        h2d.wait_stream(comp)              # earlier work on the slots comes first
        d2h.wait_stream(comp)

        def fetch(i):
            s = i % 2
            if i >= 2:
                h2d.wait_event(slot_free[s])   # state i-2's graph has read slot s
            with torch.cuda.stream(h2d):
                slot_in[s].copy_(inputs[i], non_blocking=True)
            in_ready[s].record(h2d)

        fetch(0)
        if n > 1:
            fetch(1)
        for i in range(n):
            s = i % 2
            comp.wait_event(in_ready[s])
            if i >= 2:
                comp.wait_event(out_free[s])   # state i-2's result has left output slot s
            graphs[s].replay()
            slot_free[s].record(comp)
            if i + 2 < n:
                fetch(i + 2)
            d2h.wait_event(slot_free[s])
            with torch.cuda.stream(d2h):
                outputs[i].copy_(slot_out[s], non_blocking=True)
            out_free[s].record(d2h)
        comp.wait_stream(d2h)
        # host bookkeeping as after eager steps: state and primitives agree, gradients carried
        self.cells.version += 1
        self._prims_version = self.cells.version
        self.eq._has_grads_host = True
        if st["hist"] is not None:
            self.n_hist, self.head = st["hist"]
        self.steps_done += n * steps
        return outputs

    # -- checkpoint / restart ------------------------------------------------------------------
    def state_dict(self) -> dict:
        """Everything a bitwise-identical restart needs: the conserved state, the carried limited
        gradients and their flag (the reference keeps them in ``FacetCalc.cell_grads`` and never
        saves them), the device time step, the stage / multistep history and the counters."""
        d = {"state": self.cells.state.clone(), "grads": self.eq.grads.clone(), "has_grads": self.eq.has_grads.clone(),
             "dt": self.dt.clone(), "k": self.k.clone(), "t": self.t, "steps_done": self.steps_done,
             "solver": type(self).__name__}
        d.update(self._extra_state())
        return d

    def load_state_dict(self, d: dict):
        if d.get("solver") != type(self).__name__:
            raise ValueError(f"checkpoint of a {d.get('solver')} solver, not {type(self).__name__}")
        self.cells.state = d["state"].to(self.cells.state.device)
        self.eq.grads.copy_(d["grads"])
        self.eq.has_grads.copy_(d["has_grads"])
        self.eq._has_grads_host = bool(int(d["has_grads"].item()))
        self.dt.copy_(d["dt"])
        self.k.copy_(d["k"])
        self.t, self.steps_done = d["t"], d["steps_done"]
        self._load_extra_state(d)

    def save_checkpoint(self, path: str):
        torch.save({k: (v.cpu() if isinstance(v, torch.Tensor) else v) for k, v in self.state_dict().items()}, path)

    def load_checkpoint(self, path: str):
        self.load_state_dict(torch.load(path, weights_only=False))

    def _extra_state(self) -> dict:
        return {}

    def _load_extra_state(self, d: dict):
        pass

    def _dt_changes_on_device(self) -> bool:
        tab = getattr(self, "tab", None)
        return bool(self.cfl) or bool(tab is not None and tab.adaptive)

    def solve_profile(self, warmup: int = 10, steps: int = 10, trace_path: str = "trace.json") -> str:
        """The reference's ``cfg.profile`` mode (``TSolver._solve_profile``, ``t_solvers.py:179-196``):
        ``warmup`` steps, then ``steps`` steps under ``torch.profiler`` (CPU and CUDA activity,
        shapes, stacks), the ten entries with the most CUDA time printed and a Chrome trace written
        to ``trace_path``.  Each profiled step is also an NVTX range ("fvm step <n>"), so external
        profilers can filter by it.  Returns the printed table."""
        from torch.profiler import ProfilerActivity, profile
        self.step(warmup)
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA], record_shapes=True,
                     with_stack=True, acc_events=True) as prof:      # keep every profiled step's events
            for _ in range(steps):
                prof.step()
                torch.cuda.nvtx.range_push(f"fvm step {self.steps_done}")
                self._solve_step()
                torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
        table = prof.key_averages().table(sort_by="self_cuda_time_total", row_limit=10)
        print(table)
        prof.export_chrome_trace(trace_path)
        return table

    def solve(self):
        """The reference's main loop (``TSolver._solve``, ``t_solvers.py:77-154``) on the device solver.

        Runs until ``n_iter`` steps or ``t >= end_t``.  ``t`` advances by the time step each step
        used (read from the device before the step when the step size changes on the device:
        adaptive or CFL solvers; fixed time steps need no read).  Every ``print_i`` steps: a
        progress line and a NaN check of the state.  Every ``plot_t`` of simulated time: the
        reference's NaN check of the primitives (``ValueError``; no plotting here).  With
        ``save_t`` and ``save_dir``: snapshots in the reference's ``Saver`` format, the initial
        state at t = 0 and then every ``save_t`` (``trajectory_io.TrajectorySaver``); with
        ``exact_interval`` the step that would cross a save time is shortened to land on it and
        the step size is restored afterwards.  Returns the final time.  With ``cfg.profile`` the
        reference's profiling mode runs instead (``solve_profile``)."""
        cfg = self.cfg
        if getattr(cfg, "profile", False):
            self.solve_profile()
            return self.t
        if self.n_steps is None and self.end_t is None:
            raise ValueError("Either n_iter or end_t must be set in ConfigFVM")
        saver = None
        save_t, plot_t = getattr(cfg, "save_t", None), getattr(cfg, "plot_t", None)
        if save_t and getattr(cfg, "save_dir", None) and self.n_cases == 1:
            from .trajectory_io import TrajectorySaver
            saver = TrajectorySaver(self.eq, cfg.save_dir)
            saver.save(0.0)
        exact = bool(getattr(cfg, "exact_interval", False)) and saver is not None
        read_dt = self._dt_changes_on_device()
        dt_fixed = float(self.dt[0].item())
        t, i = self.t, 0
        save_count, next_save = 1, save_t
        next_plot = 0.0
        while True:
            if self.n_steps is not None and i >= self.n_steps:
                break
            if self.end_t is not None and t >= self.end_t:
                break
            dt = float(self.dt[0].item()) if read_dt else dt_fixed
            if exact and t + dt > next_save:
                saved = self.dt.clone()
                self.dt.fill_(next_save - t)
                t = next_save
                self._solve_step()
                self.dt.copy_(saved)
            else:
                t += dt
                self._solve_step()
            if self.print_i and i % self.print_i == 0:
                if not torch.isfinite(self.cells.state).all():
                    raise ValueError("Nan detected in primatives")
                print(f"progress: i = {i}, t = {t:.4g}, dt = {dt:.3g}", flush=True)
            if plot_t and t >= next_plot:
                next_plot = t + plot_t
                if torch.isnan(self.cells.get_values()[0]).any():
                    raise ValueError("Nan detected in primatives")
            if saver is not None and t >= next_save:
                save_count += 1
                next_save = save_count * save_t
                saver.save(t)
            i += 1
        self.t = t
        return t


class Butcher(TSolver):
    def __init__(self, cells, eq, name, cfg, adaptive=False, **kw):
        self.name = name
        self.tab = make_tableau(name, adaptive=adaptive, cfl=None if adaptive else getattr(cfg, "cfl", None), **kw)
        self.n_k = self.tab.stages
        self.stages = self.tab.stages
        super().__init__(cells, eq, cfg)

    def _step(self):
        _lib.check(self._step_fn()(ct.byref(self.eq.dev.struct), ct.byref(self.eq.phys), ct.byref(self.tab),
                                   ct.byref(self.bufs), ct.byref(self.eq.work.struct), _lib.stream_ptr()),
                   "fvm_step")


class ButcherAdapt(Butcher):
    def __init__(self, cells, eq, name, cfg):
        super().__init__(cells, eq, name, cfg, adaptive=True, atol=2e-3, rtol=2e-3, mtol=1e-6,
                         alphas=(0.8, 0.995), order=4)


class RK3_SSP4(Butcher):
    def __init__(self, cells, eq, cfg):
        super().__init__(cells, eq, "RK3_SSP4", cfg, adaptive=True, b2=[0.5, 0.5, 0.0, 0.0], atol=2e-3,
                         rtol=2e-3, mtol=1e-6, alphas=(0.8, 0.995), order=4)


class AB3(TSolver):
    """Adams-Bashforth 3 (fixed dt) after two three-stage SSP-RK3 start-up steps."""
    n_k = 3
    COEF = (23 / 12, -16 / 12, 5 / 12)

    def __init__(self, cells, eq, cfg):
        self.rk = make_tableau("SSP_RK3", cfl=None)
        super().__init__(cells, eq, cfg)
        self.n_hist = 0
        self.head = 0
        self.rk_k = torch.zeros((3, eq.mesh.n_cells, eq.n_comp), device=eq.device)
        self.rk_bufs = _lib.SolverBufs(state=self.bufs.state, prims=self.bufs.prims, grads=self.bufs.grads,
                                       k=_lib.ptr(self.rk_k), dt=self.bufs.dt, has_grads=self.bufs.has_grads,
                                       cons=None)
        self._idx = (ct.c_int32 * 3)()
        self._coef = (ct.c_float * 3)()

    def _extra_state(self) -> dict:
        return {"n_hist": self.n_hist, "head": self.head, "rk_k": self.rk_k.clone()}

    def _load_extra_state(self, d: dict):
        self.n_hist, self.head = d["n_hist"], d["head"]
        self.rk_k.copy_(d["rk_k"])

    def _multistep(self, n_terms, idx, coef):
        for t in range(n_terms):
            self._idx[t] = idx[t]
            self._coef[t] = coef[t]
        fn = self.lib.fvm_multistep_fused if self.fused else self.lib.fvm_multistep
        _lib.check(fn(ct.byref(self.eq.dev.struct), ct.byref(self.eq.phys), idx[0], n_terms,
                      ct.cast(self._idx, ct.c_void_p), ct.cast(self._coef, ct.c_void_p),
                      ct.byref(self.bufs), ct.byref(self.eq.work.struct), _lib.stream_ptr()),
                   "fvm_multistep")

    def _step(self):
        h = self.head
        if self.n_hist < 2:
            # Start-up: an SSP-RK3 step from U_n; its first increment dt * f(U_n) joins the history.
            _lib.check(self._step_fn()(ct.byref(self.eq.dev.struct), ct.byref(self.eq.phys), ct.byref(self.rk),
                                       ct.byref(self.rk_bufs), ct.byref(self.eq.work.struct), _lib.stream_ptr()),
                       "fvm_step")
            self.k[h].copy_(self.rk_k[0])
        else:
            idx = [h, (h - 1) % 3, (h - 2) % 3]
            self._multistep(3, idx, list(self.COEF))
        self.n_hist = min(self.n_hist + 1, 3)
        self.head = (h + 1) % 3


def get_solver(cells, equation, cfg):
    """``get_solver`` (``integrators.py:11-27``)."""
    name, extra = cfg.solver_name, cfg.solver_extra
    if name == "RK3_SSP4":
        return RK3_SSP4(cells, equation, cfg)
    if name == "Butcher_adapt":
        return ButcherAdapt(cells, equation, extra, cfg)
    if name == "Butcher":
        return Butcher(cells, equation, extra, cfg)
    if name == "AB3":
        return AB3(cells, equation, cfg)
    if name in ("Adams3_PC", "Adams4_PC", "Euler"):
        raise NotImplementedError(f"{name} is not provided (its reference implementation cannot run)")
    raise NotImplementedError("Invalid solver.")
