"""Sparse-operator seam: ``SPM`` / ``SPMB200`` / ``to_sparse``.

Mirrors ``time_fvm/utils/sparse.py:7-70``.  ``SPMB200`` replaces ``SPMCuda`` (the Triton ELL
path): it is built once from a sparse COO/CSR matrix, packs it to ELL on the host exactly as
``csr_to_ell`` does (ascending columns per row, pad col 0 / val 0), re-lays it slot-major with
int32 columns on the device, and applies it with the CUDA kernels of ``libfvm_b200.so``.

Semantics kept from the reference:
* ``spMV(x, b)``: x 1-D [N] -> y [M]; x 2-D [N, B] -> y [M, B]; strided 1-D views are read in
  place (``ell_kernel.py:148-171``); ``b`` is added after the product.
* ``spMM(X, b)``: X [N, B] -> Y [M, B] (+ b[:, None]); B == 1 goes through the SpMV kernel.
* Outputs are newly allocated; errors are Python exceptions (``ValueError`` for ELL overflow, and
  for rows wider than 16 slots -- every operator of the residual has at most dim + 2).
* ``to_sparse(A, device)`` picks the implementation by device type.  Only CUDA devices are
  supported: there is no CPU fallback, so a non-CUDA device raises ``RuntimeError``.
"""
from __future__ import annotations

from abc import ABC, abstractmethod

import torch

from . import _lib
from .tables import coo_to_ell


class SPM(ABC):
    """Sparse matrix."""

    def __init__(self, A, device):
        self.shape = A.shape
        self.device = device

    @abstractmethod
    def spMV(self, x: torch.Tensor, b: torch.Tensor = None) -> torch.Tensor:
        """Sparse matrix-vector multiply: Ax+b"""

    @abstractmethod
    def spMM(self, X: torch.Tensor, b: torch.Tensor = None) -> torch.Tensor:
        """Sparse matrix-matrix multiply: AX+b"""


class SPMB200(SPM):
    """ELL sparse operator executed by the sm_100a kernels (``fvm_ell_spmv`` / ``fvm_ell_spmm``)."""

    def __init__(self, A: torch.Tensor, device, K: int | None = None):
        super().__init__(A, device)
        self.lib = _lib.load()
        A = A.detach().to("cpu")
        vals, cols = coo_to_ell(A if A.layout == torch.sparse_csr else A.coalesce(), K)
        if cols.numel() and int(cols.max()) >= 2 ** 31:
            raise ValueError("column index does not fit int32")
        self.M, self.K = vals.shape
        if self.K > 16:
            raise ValueError(f"ELL rows of {self.K} slots: at most 16 are supported (FVM_MAX_ELL_K)")
        self.N = A.shape[1]
        dev = torch.device(device)
        self.vals = vals.t().contiguous().to(torch.float32).to(dev)       # [K][M]
        self.cols = cols.t().contiguous().to(torch.int32).to(dev)         # [K][M]
        # row-major ELL kept as built (for inspection / bit-exactness checks)
        self.vals_rowmajor, self.cols_rowmajor = vals, cols

    def _check(self, x):
        if not x.is_cuda:
            raise RuntimeError("SPMB200 operands must be CUDA tensors")
        if x.dtype != torch.float32:
            raise TypeError(f"expected float32, got {x.dtype}")
        if x.shape[0] != self.N:
            raise ValueError(f"operand has {x.shape[0]} rows, operator has {self.N} columns")

    def spMV(self, x: torch.Tensor, b: torch.Tensor = None) -> torch.Tensor:
        self._check(x)
        if x.ndim == 2:
            return self.spMM(x, b)
        if b is not None:
            b = b.contiguous()
        y = torch.empty(self.M, device=x.device, dtype=x.dtype)
        _lib.check(self.lib.fvm_ell_spmv(_lib.ptr(self.vals), _lib.ptr(self.cols), self.M, self.K,
                                         x.data_ptr(), x.stride(0), _lib.ptr(b), _lib.ptr(y), 1,
                                         _lib.stream_ptr()), "fvm_ell_spmv")
        return y

    def spMM(self, X: torch.Tensor, b: torch.Tensor = None) -> torch.Tensor:
        self._check(X)
        if X.ndim != 2:
            raise ValueError("spMM expects a 2-D operand")
        B = X.shape[1]
        if b is not None:
            b = b.contiguous()
        if B == 1:
            y = torch.empty((self.M, 1), device=X.device, dtype=X.dtype)
            _lib.check(self.lib.fvm_ell_spmv(_lib.ptr(self.vals), _lib.ptr(self.cols), self.M, self.K,
                                             X.data_ptr(), X.stride(0), _lib.ptr(b), _lib.ptr(y), 1,
                                             _lib.stream_ptr()), "fvm_ell_spmv")
            return y
        if X.stride(1) != 1:
            X = X.contiguous()
        Y = torch.empty((self.M, B), device=X.device, dtype=X.dtype)
        _lib.check(self.lib.fvm_ell_spmm(_lib.ptr(self.vals), _lib.ptr(self.cols), self.M, self.K,
                                         X.data_ptr(), X.stride(0), B, _lib.ptr(b), _lib.ptr(Y), B,
                                         _lib.stream_ptr()), "fvm_ell_spmm")
        return Y


def to_sparse(A: torch.Tensor, device) -> SPM:
    device = torch.device(device)
    if device.type == "cuda":
        return SPMB200(A, device)
    raise RuntimeError(f"fvm_solver_b200 has no {device.type} sparse backend (CUDA only, no CPU fallback)")
