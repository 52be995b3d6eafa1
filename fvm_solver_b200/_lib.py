"""ctypes binding of ``libfvm_b200.so`` (declared in ``include/fvm_b200.h``).

The library is loaded from the package directory.  There is no fallback: if the library is
missing or CUDA is unavailable, every call raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as ct
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfvm_b200.so")

FVM_OK, FVM_E_ARG, FVM_E_CUDA, FVM_E_UNSUPPORTED, FVM_E_CAPACITY = 0, -1, -2, -3, -4
FVM_NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024
FVM_MAX_STAGES = 12
FVM_RED_DOUBLES = 64
FVM_PHASE_BC, FVM_PHASE_CELLS, FVM_PHASE_FACES, FVM_PHASE_DIV = 1, 2, 4, 8

_P = ct.c_void_p


class Mesh(ct.Structure):
    _fields_ = [(n, ct.c_int32) for n in ("dim", "n_comp", "n_cells", "n_facets", "n_bc", "n_char", "kg", "kf")] + [
        (n, _P) for n in ("cell_rec", "div_rec", "inv_h", "volumes", "face_rec",
                          "bc_cell", "bc_kind", "bc_b", "bc_l", "bc_ga", "bc_gb",
                          "bc_char", "ch_cell", "ch_normal", "ch_rho", "ch_vn", "ch_p", "ch_vt")] + [
        ("n_cases", ct.c_int32)] + [
        (n, _P) for n in ("cell_case", "face_case", "bc_case", "ch_off", "case_mu", "case_mu_b", "case_kappa")] + [
        ("n_owned", ct.c_int32), ("char_scale_given", ct.c_int32), ("case_active", _P),
        ("cell_lo", ct.c_int32), ("facet_lo", ct.c_int32)]

MESH_PTR_FIELDS = [f for f, t in Mesh._fields_ if t is _P]


class Physics(ct.Structure):
    _fields_ = [(n, ct.c_float) for n in ("T_0", "mu", "mu_b", "S_const", "C_v", "gamma", "kappa", "v_factor")] + [
        ("lim_p", ct.c_int32)]


class Work(ct.Structure):
    _fields_ = [("bc_vals", _P), ("prims", _P), ("flux", _P), ("red", _P)]


class Tableau(ct.Structure):
    _fields_ = [("stages", ct.c_int32),
                ("a", (ct.c_float * FVM_MAX_STAGES) * FVM_MAX_STAGES),
                ("b", ct.c_float * FVM_MAX_STAGES),
                ("b2", ct.c_float * FVM_MAX_STAGES),
                ("adaptive", ct.c_int32),
                ("atol", ct.c_float), ("rtol", ct.c_float), ("mtol", ct.c_float),
                ("alpha_hi_err", ct.c_float), ("alpha_lo_err", ct.c_float), ("order", ct.c_float),
                ("cfl", ct.c_float)]


class SolverBufs(ct.Structure):
    _fields_ = [(n, _P) for n in ("state", "prims", "grads", "k", "dt", "has_grads", "cons")]


_lib = None

# (name, restype, argtypes)
_SIGS = [
    ("fvm_last_cuda_error", ct.c_int, []),
    ("fvm_version", ct.c_char_p, []),
    ("fvm_ell_spmv", ct.c_int, [_P, _P, ct.c_int64, ct.c_int32, _P, ct.c_int64, _P, _P, ct.c_int64, _P]),
    ("fvm_ell_spmm", ct.c_int, [_P, _P, ct.c_int64, ct.c_int32, _P, ct.c_int64, ct.c_int32, _P, _P, ct.c_int64, _P]),
    ("fvm_residual", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), _P, _P, _P, _P, ct.POINTER(Work), _P]),
    ("fvm_stage", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), ct.POINTER(Tableau), ct.c_int32,
                             ct.POINTER(SolverBufs), ct.POINTER(Work), _P]),
    ("fvm_step", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), ct.POINTER(Tableau), ct.POINTER(SolverBufs),
                            ct.POINTER(Work), _P]),
    ("fvm_multistep", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), ct.c_int32, ct.c_int32, _P, _P,
                                 ct.POINTER(SolverBufs), ct.POINTER(Work), _P]),
    ("fvm_state_to_prims", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), _P, _P, _P]),
    ("fvm_cfl_dt", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), _P, ct.c_float, _P, ct.POINTER(Work), _P]),
    ("fvm_conservation", ct.c_int, [ct.POINTER(Mesh), _P, _P, ct.POINTER(Work), _P]),
    ("fvm_residual_noalloc", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), _P, _P, _P, _P, _P]),
    ("fvm_residual_state", ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Physics), _P, _P, _P, _P, ct.POINTER(Work), _P]),
    ("fvm_facet_values", ct.c_int, [ct.POINTER(Mesh), _P, _P, ct.POINTER(Work), _P, _P]),
    ("fvm_profile_start", ct.c_int, [ct.c_int32]),
    ("fvm_step_fused", ct.c_int, [_P, _P, _P, _P, _P, _P]),
    ("fvm_multistep_fused", ct.c_int, [_P, _P, ct.c_int32, ct.c_int32, _P, _P, _P, _P, _P]),
    ("fvm_fused_status", ct.c_int, [_P, _P]),
    ("fvm_barrier_selftest", ct.c_int, [ct.c_int32, ct.c_int32, _P]),
    ("fvm_stage_begin", ct.c_int, [_P, _P, _P, _P, _P]),
    ("fvm_stage_end", ct.c_int, [_P, _P, _P, ct.c_int32, _P, _P, ct.c_int32, _P]),
    ("fvm_stage_finalize", ct.c_int, [_P, _P, _P, _P, _P]),
    ("fvm_stage_phase", ct.c_int, [_P, _P, _P, ct.c_int32, _P, _P, ct.c_int32, ct.c_int32, _P]),
    ("fvm_char_partial", ct.c_int, [_P, _P, _P, _P, _P]),
    ("fvm_set_block_size", ct.c_int, [ct.c_int32, ct.c_int32]),
    ("fvm_set_prefetch", ct.c_int, [ct.c_int32, ct.c_int32]),
    ("fvm_set_variant", ct.c_int, [ct.c_int32, ct.c_int32]),
    ("fvm_gemm_bf16", ct.c_int, [_P, ct.c_int64, _P, ct.c_int64, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32,
                                 _P, _P, ct.c_int64, _P, _P, ct.c_int64, _P, ct.c_int32, _P, _P]),
    ("fvm_mp_gather_f32", ct.c_int, [_P, _P, ct.c_int32, ct.c_int32, _P, _P]),
    ("fvm_mp_layer", ct.c_int, [_P, _P, ct.c_int32, ct.c_int32, _P, _P, _P, _P, _P, ct.c_int32, _P, _P, _P]),
    ("fvm_mp_scatter_back", ct.c_int, [_P, _P, ct.c_int32, ct.c_int32, ct.c_int32, _P, _P, _P]),
    ("fvm_silu_back", ct.c_int, [_P, _P, ct.c_int32, ct.c_int32, _P, _P, ct.c_int64, _P, _P]),
    ("fvm_transpose_bf16", ct.c_int, [_P, ct.c_int32, ct.c_int32, ct.c_int64, _P, ct.c_int64, _P]),
    ("fvm_decoder_f32", ct.c_int, [_P, _P, _P, ct.c_int32, ct.c_int32, _P, _P]),
    ("fvm_decoder_back_f32", ct.c_int, [_P, _P, _P, ct.c_int32, ct.c_int32, _P, _P, _P, _P]),
    ("fvm_mse", ct.c_int, [_P, _P, ct.c_int64, _P, _P, _P]),
    ("fvm_adam", ct.c_int, [_P, _P, _P, _P, ct.c_int64, ct.c_float, ct.c_float, ct.c_float, ct.c_float,
                            ct.c_int32, _P, _P, ct.c_int32, ct.c_int32, _P]),
    ("fvm_corrector_features", ct.c_int, [_P, ct.c_int32, ct.c_int32, _P, _P, _P, ct.c_int32, _P, ct.c_int32, _P]),
    ("fvm_apply_increment", ct.c_int, [_P, _P, _P, ct.c_int32, ct.c_int32, _P, _P]),
    ("fvm_corrector_inputs", ct.c_int, [_P, _P, _P, _P, ct.c_int32, ct.c_int32, _P, _P, _P, ct.c_int32, _P, _P,
                                        ct.c_int32, _P]),
    ("fvm_corrector_combine", ct.c_int, [_P, _P, _P, _P, _P, _P, ct.c_int32, ct.c_int32, _P, _P]),
    ("fvm_corrector_checks", ct.c_int, [_P, _P, _P, _P, _P, _P, ct.c_int32, ct.c_int32, ct.c_int32, _P, ct.c_int32,
                                        ct.c_double, ct.c_double, ct.c_double, _P, _P, _P, _P]),
    ("fvm_set_launch_overlap", ct.c_int, [ct.c_int32]),
    ("fvm_profile_stop", ct.c_int, []),
    ("fvm_profile_read", ct.c_int, [ct.c_int32, _P, _P]),
]

KERNEL_NAMES = {0: "ell_spmv", 1: "ell_spmm", 2: "bc", 3: "cell", 4: "face", 5: "div_stage", 6: "finalize",
                7: "state_to_prims", 8: "reduce_state", 9: "batched", 10: "corrector", 11: "fused_step"}

EXPORTED = [s[0] for s in _SIGS]


def load(require_cuda: bool = True):
    """Load the library (once).  Raises if it is missing, or if CUDA is required but absent."""
    global _lib
    if require_cuda and not torch.cuda.is_available():
        raise RuntimeError("fvm_solver_b200 needs a CUDA device (B200); no CPU fallback exists")
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library {LIB_PATH} is missing; run `python -m fvm_solver_b200.build`")
        lib = ct.CDLL(LIB_PATH)
        fns = {}
        for name, res, args in _SIGS:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
            fns[name] = fn
        _lib = _Bound(fns)
    return _lib


class _Bound:
    """The library's functions, each with its declared signature.  Looking up a function that has
    no signature here raises, so no call can fall back to ctypes' default int conversion (which
    would truncate 64-bit device pointers)."""

    def __init__(self, fns: dict):
        self.__dict__.update(fns)

    def __getattr__(self, name):
        raise AttributeError(f"{name} has no declared signature in fvm_solver_b200._lib")


def check(rc: int, what: str):
    if rc != FVM_OK:
        extra = ""
        if rc == FVM_E_CUDA:
            extra = f" (cudaError {load(False).fvm_last_cuda_error()})"
        kind = {FVM_E_ARG: "invalid argument", FVM_E_CUDA: "CUDA launch failure",
                FVM_E_UNSUPPORTED: "unsupported configuration",
                FVM_E_CAPACITY: f"mesh too large for the {FVM_NOALLOC_SCRATCH_BYTES >> 20} MiB static scratch"
                }.get(rc, f"error {rc}")
        raise RuntimeError(f"{what}: {kind}{extra}")


def ptr(t) -> int | None:
    """Device pointer of a tensor (None for None / empty tensors)."""
    if t is None or t.numel() == 0:
        return None
    return t.data_ptr()


def stream_ptr(stream=None) -> int | None:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None
