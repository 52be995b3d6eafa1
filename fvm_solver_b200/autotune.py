"""Launch-configuration autotuner for the residual kernels.

The cell, facet and divergence kernels (one thread per cell / facet) run at any block size, with or
without the L2 prefetch of their record streams one wave of blocks ahead; which configuration is
fastest depends on the mesh (cell count, boundary fraction, batched or not) because it sets how
many warps each SM keeps in flight against the gather latency and whether the records still come
from DRAM when a block reads them.  ``autotune`` times each candidate (block size, prefetch) on the
caller's own mesh -- residual evaluations bracketed by the library's per-launch CUDA events --
keeps the fastest per kernel, and installs it with ``fvm_set_block_size`` / ``fvm_set_prefetch``
(for the facet kernel also the record-staging variant, ``fvm_set_variant``).
Results do not change with either (every thread's arithmetic is the same), only the time does.
Choices are cached per (dim, cell-count bucket, batch size).
"""
from __future__ import annotations

import ctypes as ct
import math

import numpy as np
import torch

from . import _lib

CANDIDATES = (64, 128, 256, 512)
PREFETCH = (0, 1)           # off, one wave of resident blocks ahead
KERNELS = {3: "cell", 4: "face", 5: "div_stage"}
_cache: dict = {}


def _key(eq) -> tuple:
    n = eq.mesh.n_cells
    return (eq.mesh.dim, int(round(math.log2(max(n, 1)) * 2)), int(getattr(eq, "n_cases", 0) or 0))


def set_block_size(kernel: str, threads: int):
    kid = {v: k for k, v in KERNELS.items()}[kernel]
    _lib.check(_lib.load().fvm_set_block_size(kid, int(threads)), "fvm_set_block_size")


def set_prefetch(kernel: str, blocks_ahead: int):
    kid = {v: k for k, v in KERNELS.items()}[kernel]
    _lib.check(_lib.load().fvm_set_prefetch(kid, int(blocks_ahead)), "fvm_set_prefetch")


def set_variant(kernel: str, variant: int):
    kid = {v: k for k, v in KERNELS.items()}[kernel]
    _lib.check(_lib.load().fvm_set_variant(kid, int(variant)), "fvm_set_variant")


def set_launch_overlap(on: bool):
    """Programmatic dependent launches for the stage kernels (``fvm_set_launch_overlap``; on by
    default): each kernel is launched while its predecessor drains and waits on the device."""
    _lib.check(_lib.load().fvm_set_launch_overlap(int(bool(on))), "fvm_set_launch_overlap")


STAGED = "staged"           # facet kernel: records staged in shared memory by the bulk-copy unit


def _install(kernel: str, cfg: tuple):
    set_block_size(kernel, cfg[0])
    if cfg[1] == STAGED:
        set_prefetch(kernel, 0)
        set_variant(kernel, 1)
        return
    set_prefetch(kernel, cfg[1])
    if kernel == "face":
        set_variant(kernel, 0)


def _time_residual(eq, prims, out, reps: int) -> dict:
    """Mean device time per launch of each kernel over ``reps`` residual evaluations."""
    lib = eq.lib
    _lib.check(lib.fvm_profile_start(reps * 8 + 8), "fvm_profile_start")
    for _ in range(reps):
        _lib.check(lib.fvm_residual(ct.byref(eq.dev.struct), ct.byref(eq.phys), _lib.ptr(prims), _lib.ptr(eq.grads),
                                    _lib.ptr(eq.has_grads), _lib.ptr(out), ct.byref(eq.work.struct),
                                    _lib.stream_ptr()), "fvm_residual")
    n = lib.fvm_profile_stop()
    if n < 0:
        raise RuntimeError("profiling buffer overflow")
    ids = np.zeros(n, np.int32)
    ms = np.zeros(n, np.float32)
    if lib.fvm_profile_read(n, ids.ctypes.data, ms.ctypes.data) != n:
        raise RuntimeError("fvm_profile_read failed")
    return {KERNELS[k]: float(ms[ids == k].mean()) for k in KERNELS if np.any(ids == k)}


def autotune(eq, reps: int = 5, candidates=CANDIDATES, prefetch=PREFETCH, use_cache: bool = True,
             staged: bool = True, owner: bool = True) -> dict:
    """Pick and install the fastest (block size, prefetch) per kernel for ``eq`` (FVMEquation or
    BatchedFVM).

    The carried limited gradients are saved and restored, so the tuning runs leave the solver's
    state untouched.  Returns ``{kernel: {"threads": bs, "prefetch": pf, "ms": {(bs, pf): mean ms}}}``.
    With ``owner``, residual evaluations then time the owner-computes divergence (each cell
    evaluates its own facets' fluxes, no flux array) against facet kernel + divergence kernel and
    keep the faster (``best["div_stage"]["residual_variant"]``: 1 owner computes, 0 separate).
    """
    key = _key(eq)
    if use_cache and key in _cache:
        for k, v in _cache[key].items():
            _install(k, v["cfg"])
        set_variant("div_stage", _cache[key]["div_stage"].get("residual_variant", 0))
        return _cache[key]
    prims = eq.cells.get_values()[0].contiguous()
    out = torch.empty_like(prims)
    g_save, f_save = eq.grads.clone(), eq.has_grads.clone()
    timings = {k: {} for k in KERNELS.values()}
    set_variant("div_stage", 0)                             # the per-kernel timings need the facet kernel
    for bs in candidates:
        for pf in tuple(prefetch) + ((STAGED,) if staged else ()):
            for k in KERNELS.values():
                _install(k, (bs, pf if (pf != STAGED or k == "face") else 0))
            _time_residual(eq, prims, out, 1)               # warm-up at this configuration
            for k, ms in _time_residual(eq, prims, out, reps).items():
                if pf == STAGED and k != "face":
                    continue
                timings[k][(bs, pf)] = ms
    best = {}
    for k, t in timings.items():
        cfg = min(t, key=t.get)
        best[k] = {"threads": cfg[0], "prefetch": 0 if cfg[1] == STAGED else cfg[1],
                   "variant": "staged" if cfg[1] == STAGED else "registers", "cfg": cfg,
                   "ms": {f"{a}/{b}": v for (a, b), v in t.items()}}
        _install(k, cfg)
    set_variant("div_stage", 0)
    if owner:
        sep = _time_residual(eq, prims, out, reps)
        t_sep = sep.get("face", 0.0) + sep.get("div_stage", 0.0)
        set_variant("div_stage", 1)
        _time_residual(eq, prims, out, 1)
        t_own = _time_residual(eq, prims, out, reps).get("div_stage", float("inf"))
        variant = 1 if t_own < t_sep else 0
        set_variant("div_stage", variant)
        best["div_stage"]["residual_variant"] = variant
        best["div_stage"]["residual_ms"] = {"separate": t_sep, "owner_computes": t_own}
    eq.grads.copy_(g_save)
    eq.has_grads.copy_(f_save)
    torch.cuda.synchronize()
    _cache[key] = best
    return best


def reset():
    """Back to the defaults (256 threads, no prefetch, per-thread record loads, separate facet and
    divergence kernels) for every tunable kernel."""
    for k in KERNELS.values():
        _install(k, (256, 0))
    set_variant("div_stage", 0)


def tune_fused(eq, steps: int = 10, reps: int = 3) -> dict:
    """Choose between separate launches per phase and the fused cooperative step for ``eq``'s
    time stepper: each variant's CUDA graph of ``steps`` steps is replayed ``reps`` times on a copy
    of the state, timed with CUDA events; the faster is kept (``t_solver.fused``).  The solver's
    state, carried gradients, dt and history are restored.  Returns {"fused": bool, "ms": {...}}."""
    sol = eq.t_solver
    saved = sol.state_dict()
    times = {}
    for fused in (False, True):
        sol.fused = fused
        replay = sol.graph_steps(steps)
        replay()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            replay()
        e1.record()
        torch.cuda.synchronize()
        times[fused] = e0.elapsed_time(e1) / (reps * steps)
        del replay
        sol.load_state_dict(saved)
    sol.fused = times[True] < times[False]
    if sol.fused_status():
        raise RuntimeError("fused step: a grid barrier wait gave up")
    return {"fused": sol.fused, "ms_per_step": {"separate": times[False], "fused": times[True]}}
