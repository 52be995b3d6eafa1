"""Learned k-step corrector with plain-FVM fallback.

A small message-passing network over the mesh's face adjacency predicts the state change over
k FVM steps; a proposal is accepted only if it passes two checks against the FVM itself, else the
window is recomputed with k plain FVM steps.

Network (width W = 64, L = 4 message-passing layers, SiLU):
    X  = [normalised state, geometry, case parameters]            (bf16 [N][64])
    h0 = SiLU(X Win^T + b_in)
    h_{l+1} = h_l + SiLU([h_l, mean_{j in nbr} h_l,j] W_l^T + b_l)  (l = 0..3)
    out = h_L Wout^T + b_out                                        (normalised dU over k steps)
All matrix products run on ``fvm_gemm_bf16`` (tcgen05, BF16 operands, FP32 accumulation in tensor
memory, bias / SiLU / residual fused into the epilogue); the backward pass (SiLU derivative,
transposed products, split-K weight gradients, the transpose of the neighbour mean) and Adam are
the library's own kernels as well.  Weights are kept in FP32 (master) with BF16 copies for the GEMMs.

Training data are trajectories the batched FVM solver generates (``BatchedFVM``): every step of a
spin-up-then-record run is stored on the device and random (U_t, U_{t+k}) windows are drawn.

Fallback (per case, per window): the proposal U' = U + scale * net(U) is accepted when
  * the relative mass / energy drift |M(U') - M(U) - k dt sum(vol dU/dt(U))| / |M(U)| <= 1e-4
    (the expected change is the FVM boundary-flux integral over the window, so open channels are
    judged correctly), and
  * ||dU/dt(U')||_vol <= 3 ||dU/dt(U)||_vol;
otherwise the window is advanced with k plain FVM steps.
"""
from __future__ import annotations

import ctypes as ct
import math
import time

import numpy as np
import torch

from . import _lib

W = 64
XW = 64


def _bf(t):
    return t.to(torch.bfloat16).contiguous()


def neighbour_table(kt) -> torch.Tensor:
    """[N][K] int32 face neighbours of each cell (-1 for boundary faces), from the gradient stencil."""
    N = kt.n_cells
    cols = kt.g_cols.t().long()                    # [N][kg]
    own = torch.arange(N).unsqueeze(1)
    nb = torch.where((cols != own) & (cols < N), cols, torch.full_like(cols, -1))
    # keep the first dim+1 neighbour slots (a cell has at most dim+1 face neighbours)
    nb, _ = torch.sort(nb, dim=1, descending=True)
    return nb[:, :kt.dim + 1].contiguous().to(torch.int32)


def geometry_features(kt, case_params: torch.Tensor | None, lengths=(2.0, 1.0)) -> torch.Tensor:
    """Per-cell static features: centroid / domain size, standardised log volume, centroid->facet
    vectors / sqrt(volume), and per-case parameters (Mach, log10 Re) broadcast to the cells."""
    N, dim = kt.n_cells, kt.dim
    cen = kt.centroids.double() / torch.tensor(lengths[:dim], dtype=torch.float64)
    lv = torch.log(kt.volumes)
    lv = (lv - lv.mean()) / (lv.std() + 1e-12)
    scale = kt.volumes.sqrt().unsqueeze(1) if dim == 2 else kt.volumes.pow(1.0 / 3.0).unsqueeze(1)
    disp = kt.disp.permute(2, 0, 1).reshape(N, -1).double() / scale
    feats = [cen, lv.unsqueeze(1), disp]
    if case_params is not None:
        feats.append(case_params.double())
    return torch.cat(feats, 1).float().contiguous()


class CorrectorNet:
    """Parameters, forward, backward and Adam of the message-passing corrector (see module doc)."""

    def __init__(self, n_out: int, layers: int = 4, device="cuda", seed: int = 0, lr: float = 1e-3):
        self.lib = _lib.load()
        self.dev = torch.device(device)
        self.L, self.O, self.lr = layers, n_out, lr
        g = torch.Generator().manual_seed(seed)
        U = lambda shape, fan: ((torch.rand(shape, generator=g) * 2 - 1) * math.sqrt(3.0 / fan)).to(self.dev)
        self.params = {"W_in": U((W, XW), XW), "b_in": torch.zeros(W, device=self.dev)}
        for l in range(layers):
            self.params[f"W{l}"] = U((W, 2 * W), 2 * W) * 0.5
            self.params[f"b{l}"] = torch.zeros(W, device=self.dev)
        self.params["W_out"] = U((n_out, W), W) * 0.1
        self.params["b_out"] = torch.zeros(n_out, device=self.dev)
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.bf = {k: _bf(self.params[k]) for k in ["W_in"] + [f"W{l}" for l in range(layers)]}
        self.bfT = {f"W{l}": _bf(self.params[f"W{l}"].t()) for l in range(layers)}
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self._bufs = None

    # -- buffers ---------------------------------------------------------------------------------
    def _alloc(self, N: int):
        if self._bufs is not None and self._bufs["N"] == N:
            return self._bufs
        Np = (N + 63) // 64 * 64
        d, L = self.dev, self.L
        b = {"N": N, "Np": Np,
             "X": torch.zeros((Np, XW), dtype=torch.bfloat16, device=d),
             "XT": torch.zeros((XW, Np), dtype=torch.bfloat16, device=d),
             "Z": [torch.zeros((N, W), device=d) for _ in range(L + 1)],
             "hf": [torch.zeros((N, W), device=d) for _ in range(L + 1)],
             "hb": [torch.zeros((Np, W), dtype=torch.bfloat16, device=d) for _ in range(L + 1)],
             "A": [torch.zeros((Np, 2 * W), dtype=torch.bfloat16, device=d) for _ in range(L)],
             "AT": torch.zeros((2 * W, Np), dtype=torch.bfloat16, device=d),
             "dZ": torch.zeros((Np, W), dtype=torch.bfloat16, device=d),
             "dZT": torch.zeros((W, Np), dtype=torch.bfloat16, device=d),
             "dA": torch.zeros((N, 2 * W), device=d),
             "dh": torch.zeros((N, W), device=d), "dh2": torch.zeros((N, W), device=d),
             "out": torch.zeros((N, self.O), device=d), "dout": torch.zeros((N, self.O), device=d),
             "loss": torch.zeros(1, dtype=torch.float64, device=d)}
        self._bufs = b
        return b

    def _gemm(self, A, lda, B, ldb, M, N, K, Df=None, Db=None, ldd=0, bias=None, resid=None, ldr=0, pre=None,
              act=0, k_splits=1):
        _lib.check(self.lib.fvm_gemm_bf16(A.data_ptr(), lda, B.data_ptr(), ldb, M, N, K, k_splits, _lib.ptr(bias),
                                          _lib.ptr(resid), ldr, _lib.ptr(Df), _lib.ptr(Db), ldd, _lib.ptr(pre),
                                          act, self.err.data_ptr(), _lib.stream_ptr()), "fvm_gemm_bf16")

    # -- forward ---------------------------------------------------------------------------------
    def features(self, state, mean, inv_std, geo):
        b = self._alloc(state.shape[0])
        N, C = state.shape
        _lib.check(self.lib.fvm_corrector_features(state.data_ptr(), N, C, mean.data_ptr(), inv_std.data_ptr(),
                                                   geo.data_ptr(), geo.shape[1], b["X"].data_ptr(), XW,
                                                   _lib.stream_ptr()), "fvm_corrector_features")
        return b["X"]

    def forward(self, nbr: torch.Tensor) -> torch.Tensor:
        """Network output for the features already in the X buffer (``features``)."""
        b = self._bufs
        N, L = b["N"], self.L
        p, s = self.params, _lib.stream_ptr()
        self._gemm(b["X"], XW, self.bf["W_in"], XW, N, W, XW, Df=b["hf"][0], Db=b["hb"][0], ldd=W, bias=p["b_in"],
                   pre=b["Z"][0], act=1)
        for l in range(L):
            _lib.check(self.lib.fvm_mp_gather(b["hb"][l].data_ptr(), nbr.data_ptr(), N, W, nbr.shape[1],
                                              b["A"][l].data_ptr(), s), "fvm_mp_gather")
            self._gemm(b["A"][l], 2 * W, self.bf[f"W{l}"], 2 * W, N, W, 2 * W, Df=b["hf"][l + 1], Db=b["hb"][l + 1],
                       ldd=W, bias=p[f"b{l}"], resid=b["hf"][l], ldr=W, pre=b["Z"][l + 1], act=1)
        _lib.check(self.lib.fvm_decoder(b["hb"][L].data_ptr(), p["W_out"].data_ptr(), p["b_out"].data_ptr(), N, W,
                                        self.O, b["out"].data_ptr(), s), "fvm_decoder")
        return b["out"]

    # -- backward + optimiser --------------------------------------------------------------------
    def train_step(self, nbr: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        """One Adam step on the MSE between the network output and ``target`` [N][O].

        Returns the loss as a device tensor (no host synchronisation)."""
        b = self._bufs
        N, Np, L, s = b["N"], b["Np"], self.L, _lib.stream_ptr()
        p, g = self.params, self.grads
        self.forward(nbr)
        b["loss"].zero_()
        _lib.check(self.lib.fvm_mse(b["out"].data_ptr(), target.data_ptr(), N * self.O, b["loss"].data_ptr(),
                                    b["dout"].data_ptr(), s), "fvm_mse")
        _lib.check(self.lib.fvm_decoder_back(b["hb"][L].data_ptr(), p["W_out"].data_ptr(), b["dout"].data_ptr(), N,
                                             W, self.O, b["dh"].data_ptr(), g["W_out"].data_ptr(),
                                             g["b_out"].data_ptr(), s), "fvm_decoder_back")
        dh, dh2 = b["dh"], b["dh2"]
        splits = max(1, min(512, (Np // 64) // 8))
        for l in reversed(range(L)):
            _lib.check(self.lib.fvm_silu_back(dh.data_ptr(), b["Z"][l + 1].data_ptr(), N, W, b["dZ"].data_ptr(),
                                              b["dZT"].data_ptr(), Np, g[f"b{l}"].data_ptr(), s), "fvm_silu_back")
            _lib.check(self.lib.fvm_transpose_bf16(b["A"][l].data_ptr(), N, 2 * W, 2 * W, b["AT"].data_ptr(), Np, s),
                       "fvm_transpose_bf16")
            # dW_l += dZ^T A_l   (M = 64 output channels, N = 128 inputs, K = cells, split-K)
            self._gemm(b["dZT"], Np, b["AT"], Np, W, 2 * W, Np, Df=g[f"W{l}"], ldd=2 * W, k_splits=splits)
            # dA = dZ W_l
            self._gemm(b["dZ"], W, self.bfT[f"W{l}"], W, N, 2 * W, W, Df=b["dA"], ldd=2 * W)
            # dh_l = dh_{l+1} (residual) + dA[:, :W] + transpose of the neighbour mean of dA[:, W:]
            _lib.check(self.lib.fvm_mp_scatter_back(b["dA"].data_ptr(), nbr.data_ptr(), N, W, nbr.shape[1],
                                                    dh.data_ptr(), dh2.data_ptr(), s), "fvm_mp_scatter_back")
            dh, dh2 = dh2, dh
        _lib.check(self.lib.fvm_silu_back(dh.data_ptr(), b["Z"][0].data_ptr(), N, W, b["dZ"].data_ptr(),
                                          b["dZT"].data_ptr(), Np, g["b_in"].data_ptr(), s), "fvm_silu_back")
        _lib.check(self.lib.fvm_transpose_bf16(b["X"].data_ptr(), N, XW, XW, b["XT"].data_ptr(), Np, s),
                   "fvm_transpose_bf16")
        self._gemm(b["dZT"], Np, b["XT"], Np, W, XW, Np, Df=g["W_in"], ldd=XW, k_splits=splits)
        self.adam()
        return b["loss"]

    def adam(self, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        s = _lib.stream_ptr()
        for k, prm in self.params.items():
            pb = self.bf.get(k)
            pbT = self.bfT.get(k)
            rows, cols = (prm.shape[0], prm.shape[1]) if prm.ndim == 2 else (1, prm.shape[0])
            _lib.check(self.lib.fvm_adam(prm.data_ptr(), self.grads[k].data_ptr(), self.m[k].data_ptr(),
                                         self.v[k].data_ptr(), prm.numel(), self.lr, beta1, beta2, eps,
                                         self.step_count, _lib.ptr(pb), _lib.ptr(pbT), rows, cols, s), "fvm_adam")

    def check_errors(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("tensor-core completion wait timed out in fvm_gemm_bf16")


# ---------------------------------------------------------------------------------------------
# Training on solver trajectories and corrected rollouts
# ---------------------------------------------------------------------------------------------
class CorrectorModel:
    """Network + the normalisation and geometry of one batch of meshes."""

    def __init__(self, batch, case_params: torch.Tensor, k: int = 8, seed: int = 0, lr: float = 1e-3,
                 like: "CorrectorModel | None" = None):
        """``like``: reuse another model's trained network and normalisation on this batch of meshes
        (the weights are mesh-independent; neighbours and geometry are this batch's)."""
        self.batch = batch
        self.k = k if like is None else like.k
        C = batch.n_comp
        kt = batch.kt
        self.net = CorrectorNet(C, device=batch.device, seed=seed, lr=lr) if like is None else like.net
        self.nbr = neighbour_table(kt).to(batch.device)
        cp = case_params[batch.dev.case["cell_case"].long().cpu()]
        self.geo = geometry_features(kt, cp).to(batch.device)
        if C + self.geo.shape[1] > XW:
            raise ValueError("too many input features")
        self.mean = torch.zeros(C, device=batch.device)
        self.inv_std = torch.ones(C, device=batch.device)
        self.scale = torch.ones(C, device=batch.device)
        if like is not None:
            self.mean, self.inv_std, self.scale = like.mean, like.inv_std, like.scale

    def set_normalisation(self, states: torch.Tensor, increments: torch.Tensor):
        self.mean = states.mean(dim=(0, 1)).float().contiguous()
        self.inv_std = (1.0 / (states.std(dim=(0, 1)) + 1e-6)).float().contiguous()
        self.scale = (increments.std(dim=(0, 1)) + 1e-12).float().contiguous()

    def predict(self, state: torch.Tensor, out_state: torch.Tensor):
        self.net.features(state, self.mean, self.inv_std, self.geo)
        out = self.net.forward(self.nbr)
        N, C = state.shape
        lib = self.net.lib
        _lib.check(lib.fvm_apply_increment(state.data_ptr(), out.data_ptr(), self.scale.data_ptr(), N, C,
                                           out_state.data_ptr(), _lib.stream_ptr()), "fvm_apply_increment")
        return out_state


def record_trajectory(batch, steps: int, spinup: int) -> torch.Tensor:
    """Advance ``batch`` ``spinup`` steps, then record ``steps + 1`` states on the device."""
    sol = batch.t_solver
    sol.step(spinup)
    traj = torch.empty((steps + 1, *batch.cells.state.shape), device=batch.device)
    traj[0].copy_(batch.cells.state)
    for t in range(steps):
        sol.step(1)
        traj[t + 1].copy_(batch.cells.state)
    return traj


def train(model: CorrectorModel, traj: torch.Tensor, iters: int, seed: int = 0, log_every: int = 0) -> list:
    """Adam on random windows (U_t -> U_{t+k}) of a recorded trajectory; returns the loss history."""
    k = model.k
    T = traj.shape[0] - k
    inc = traj[k:] - traj[:T]
    model.set_normalisation(traj, inc)
    g = torch.Generator().manual_seed(seed)
    target = torch.empty_like(traj[0])
    losses = []
    model.net._alloc(traj.shape[1])
    for it in range(iters):
        t = int(torch.randint(0, T, (1,), generator=g))
        torch.div(inc[t], model.scale, out=target)
        model.net.features(traj[t], model.mean, model.inv_std, model.geo)
        loss = model.net.train_step(model.nbr, target)
        if log_every and (it % log_every == 0 or it == iters - 1):
            losses.append((it, float(loss.item())))
    model.net.check_errors()
    return losses


class CheckedRollout:
    """Corrector + fallback rollout on a batch, with per-case acceptance checks (see module doc)."""

    def __init__(self, model: CorrectorModel, drift_tol: float = 1e-4, residual_ratio: float = 3.0):
        self.m = model
        b = model.batch
        self.b = b
        self.lib = _lib.load()
        self.drift_tol, self.ratio = drift_tol, residual_ratio
        N, C = b.cells.state.shape
        d = b.device
        self.prop = torch.empty((N, C), device=d)
        self.r0 = torch.empty((N, C), device=d)
        self.r1 = torch.empty((N, C), device=d)
        self.sq = torch.empty((N, C), device=d)
        self.grads = torch.zeros_like(b.grads)
        self.flag = torch.zeros(1, dtype=torch.int32, device=d)
        self.cons = torch.empty((b.n_cases, C), dtype=torch.float64, device=d)
        self.accepted = 0
        self.windows = 0

    def _residual(self, state, out):
        prims = self.b.cells.phys_setup.state_to_primative(state)[0].contiguous()
        self.flag.zero_()
        _lib.check(self.lib.fvm_residual(ct.byref(self.b.dev.struct), ct.byref(self.b.phys), prims.data_ptr(),
                                         self.grads.data_ptr(), self.flag.data_ptr(), out.data_ptr(),
                                         ct.byref(self.b.work.struct), _lib.stream_ptr()), "fvm_residual")

    def _sums(self, x) -> torch.Tensor:
        out = torch.empty((self.b.n_cases, x.shape[1]), dtype=torch.float64, device=x.device)
        _lib.check(self.lib.fvm_conservation(ct.byref(self.b.dev.struct), x.contiguous().data_ptr(), out.data_ptr(),
                                             ct.byref(self.b.work.struct), _lib.stream_ptr()), "fvm_conservation")
        return out

    def window(self) -> torch.Tensor:
        """Advance one window of k steps; returns the per-case acceptance mask (device)."""
        b, k = self.b, self.m.k
        U = b.cells.state
        dim = b.mesh.dim
        self._residual(U, self.r0)
        self.m.predict(U, self.prop)
        self._residual(self.prop, self.r1)
        M0, Mp, R0 = self._sums(U), self._sums(self.prop), self._sums(self.r0)
        dt = b.t_solver.dt.double()
        cons = [dim, dim + 1]                                # mass and energy
        expected = M0[:, cons] + k * dt[:, None] * R0[:, cons]
        drift = ((Mp[:, cons] - expected).abs() / M0[:, cons].abs()).max(dim=1).values
        torch.mul(self.r0, self.r0, out=self.sq)
        n0 = self._sums(self.sq).sum(dim=1)
        torch.mul(self.r1, self.r1, out=self.sq)
        n1 = self._sums(self.sq).sum(dim=1)
        ok = (drift <= self.drift_tol) & (n1 <= self.ratio ** 2 * n0) & torch.isfinite(drift)
        self.windows += b.n_cases
        if bool(ok.all()):
            b.cells.state = self.prop
            self.accepted += b.n_cases
            return ok
        # fallback: k plain FVM steps for the batch, then keep the accepted proposals
        keep = ok[b.dev.case["cell_case"].long()].unsqueeze(1)
        b.t_solver.step(k)
        b.cells.state = torch.where(keep, self.prop, b.cells.state)
        self.accepted += int(ok.sum())
        return ok
