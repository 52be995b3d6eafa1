"""Learned k-step corrector with plain-FVM fallback.

A small message-passing network over the mesh's face adjacency corrects a first-order estimate of
the state change over k FVM steps; a proposal is accepted only if it passes two checks against the
FVM itself, else the window is recomputed with k plain FVM steps.

Proposal for a window starting at U (per case time step dt, R = the FVM residual dU/dt):
    base = k dt R(U)                                     (k forward-Euler steps of the FVM residual)
    U'   = U + base + P(scale * net([U, base], geometry))
where P removes, per case, the volume-weighted mean of the mass and energy components of the
learned part, so the proposal changes total mass and energy by exactly k dt sum(vol R(U)) -- the
FVM boundary-flux integral over the window.  The network only has to learn the higher-order part of
the k-step change, and the conservation check cannot be failed by the network.

Network (width W = 64, L = 4 message-passing layers, SiLU):
    X  = [normalised U, normalised base, geometry, case parameters]   (bf16 [N][64])
    h0 = SiLU(X Win^T + b_in)                                        (h: fp32 residual stream)
    h_{l+1} = h_l + SiLU([bf16(h_l), bf16(mean_{j in nbr} h_l,j)] W_l^T + b_l)  (l = 0..3)
    out = h_L Wout^T + b_out                                        (normalised U_{t+k} - U_t - base)
All matrix products run on ``fvm_gemm_bf16`` (tcgen05, BF16 operands, FP32 accumulation in tensor
memory, bias / SiLU / residual fused into the epilogue); the backward pass (SiLU derivative,
transposed products, split-K weight gradients, the transpose of the neighbour mean) and Adam are
the library's own kernels as well.  Weights are kept in FP32 (master) with BF16 copies for the GEMMs.

Training data are trajectories the batched FVM solver generates (``BatchedFVM``): every step of a
spin-up-then-record run is stored on the device and random (U_t, U_{t+k}) windows are drawn.

Fallback (per case, per window): the proposal U' is accepted when
  * the relative mass / energy drift |M(U') - M(U) - k dt sum(vol dU/dt(U))| / |M(U)| <= 1e-4,
  * ||dU/dt(U')||_vol <= 3 ||dU/dt(U)||_vol, and
  * U' is admissible: positive density and internal energy in every cell;
otherwise the case is advanced with k plain FVM steps.  The proposal and the checks are one CUDA
graph; the host reads the per-case verdicts once per window and, when some case failed, replays a
graph of k FVM steps with the accepted cases frozen (``BatchedFVM.use_case_mask``: the kernels skip
their cells, facets and boundary facets), so the fallback costs in proportion to the failed cases.
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


def _group_world(group) -> int:
    import torch.distributed as dist
    return dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1


def broadcast_from_first(tensors, group=None):
    """Overwrite ``tensors`` on every rank of ``group`` with the first rank's values (no-op on one
    rank)."""
    import torch.distributed as dist
    if _group_world(group) == 1:
        return
    src = dist.get_global_rank(group, 0) if group is not None else 0
    for t in tensors:
        dist.broadcast(t, src=src, group=group)


class GradBucket:
    """Data-parallel gradient exchange: the gradients of all parameters live in one flat buffer
    (``views`` holds one view per parameter), so a training iteration averages them over the ranks
    of ``group`` with a single all-reduce (NCCL between GPUs, gloo on CPU) before the optimiser
    step.  With one rank (or no process group) ``average`` does nothing."""

    def __init__(self, tensors: dict):
        first = next(iter(tensors.values()))
        total = sum(t.numel() for t in tensors.values())
        self.flat = torch.zeros(total, dtype=first.dtype, device=first.device)
        self.views, o = {}, 0
        for k, t in tensors.items():
            v = self.flat[o:o + t.numel()].view(t.shape)
            v.copy_(t)
            self.views[k] = v
            o += t.numel()
        self.group = None
        self.world = 1

    def attach(self, group=None):
        self.group = group
        self.world = _group_world(group)

    def average(self):
        if self.world == 1:
            return
        import torch.distributed as dist
        dist.all_reduce(self.flat, op=dist.ReduceOp.SUM, group=self.group)
        self.flat.div_(self.world)


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
        self.bucket = GradBucket({k: torch.zeros_like(v) for k, v in self.params.items()})
        self.grads = self.bucket.views
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

    def forward(self, nbr: torch.Tensor, store_pre: bool = True) -> torch.Tensor:
        """Network output for the features already in the X buffer (``features``).

        Training (``store_pre=True``): the input GEMM, then per layer the gather of
        [bf16(h_i), bf16(mean_j h_j)] from the fp32 residual stream (kept for the backward pass)
        and a GEMM whose epilogue adds bias, SiLU and the residual, storing the pre-activations;
        the decoder reads the last fp32 activations.  Inference (``store_pre=False``): the input
        GEMM, then one persistent fused kernel per layer (``fvm_mp_layer``: the gather built in
        shared memory, tcgen05 MMA, epilogue), the last one with the decoder in its epilogue.  Both
        forms do the same arithmetic in the same order and give bitwise the same output."""
        b = self._bufs
        N, L = b["N"], self.L
        p, s = self.params, _lib.stream_ptr()
        Z = b["Z"] if store_pre else [None] * (L + 1)
        self._gemm(b["X"], XW, self.bf["W_in"], XW, N, W, XW, Df=b["hf"][0], ldd=W, bias=p["b_in"], pre=Z[0], act=1)
        for l in range(L):
            if not store_pre:
                last = l == L - 1
                _lib.check(self.lib.fvm_mp_layer(b["hf"][l].data_ptr(), nbr.data_ptr(), N, nbr.shape[1],
                                                 self.bf[f"W{l}"].data_ptr(), p[f"b{l}"].data_ptr(),
                                                 None if last else b["hf"][l + 1].data_ptr(),
                                                 p["W_out"].data_ptr() if last else None,
                                                 p["b_out"].data_ptr() if last else None, self.O,
                                                 b["out"].data_ptr() if last else None, self.err.data_ptr(), s),
                           "fvm_mp_layer")
                continue
            _lib.check(self.lib.fvm_mp_gather_f32(b["hf"][l].data_ptr(), nbr.data_ptr(), N, nbr.shape[1],
                                                  b["A"][l].data_ptr(), s), "fvm_mp_gather_f32")
            self._gemm(b["A"][l], 2 * W, self.bf[f"W{l}"], 2 * W, N, W, 2 * W, Df=b["hf"][l + 1], ldd=W,
                       bias=p[f"b{l}"], resid=b["hf"][l], ldr=W, pre=Z[l + 1], act=1)
        if store_pre:
            _lib.check(self.lib.fvm_decoder_f32(b["hf"][L].data_ptr(), p["W_out"].data_ptr(), p["b_out"].data_ptr(),
                                                N, self.O, b["out"].data_ptr(), s), "fvm_decoder_f32")
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
        _lib.check(self.lib.fvm_decoder_back_f32(b["hf"][L].data_ptr(), p["W_out"].data_ptr(), b["dout"].data_ptr(),
                                                 N, self.O, b["dh"].data_ptr(), g["W_out"].data_ptr(),
                                                 g["b_out"].data_ptr(), s), "fvm_decoder_back_f32")
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
        self.bucket.average()
        self.adam()
        return b["loss"]

    def data_parallel(self, group=None):
        """Train data-parallel over the ranks of ``group`` (one process per GPU): the first rank's
        weights are broadcast, and every ``train_step`` averages the gradients of all ranks (one
        all-reduce of the flat gradient buffer) before Adam, so the ranks' weights stay identical."""
        self.bucket.attach(group)
        broadcast_from_first(list(self.params.values()), group)
        for k in self.bf:
            self.bf[k].copy_(_bf(self.params[k]))
        for k in self.bfT:
            self.bfT[k].copy_(_bf(self.params[k].t()))
        return self

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

    def state_dict(self) -> dict:
        """FP32 master weights and the layer count (the Adam moments are not kept)."""
        return {"layers": self.L, "n_out": self.O, "params": {k: v.detach().cpu().clone() for k, v in self.params.items()}}

    def load_state_dict(self, d: dict):
        if d["layers"] != self.L or d["n_out"] != self.O:
            raise ValueError("checkpoint network shape differs")
        for k, v in d["params"].items():
            self.params[k].copy_(v.to(self.dev))
        for k in self.bf:
            self.bf[k].copy_(_bf(self.params[k]))
        for k in self.bfT:
            self.bfT[k].copy_(_bf(self.params[k].t()))

    def check_errors(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("tensor-core completion wait timed out in fvm_gemm_bf16")


# ---------------------------------------------------------------------------------------------
# Training on solver trajectories and corrected rollouts
# ---------------------------------------------------------------------------------------------
class ResidualEval:
    """dU/dt of a batch for a given conserved state, on scratch gradients (the solver's carried
    gradients are left alone), as the FVM residual of the first stage of a fresh run."""

    def __init__(self, batch):
        self.b = batch
        self.lib = _lib.load()
        self.grads = torch.zeros_like(batch.grads)
        self.flag = torch.zeros(1, dtype=torch.int32, device=batch.device)

    def __call__(self, state: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        self.flag.zero_()
        _lib.check(self.lib.fvm_residual_state(ct.byref(self.b.dev.struct), ct.byref(self.b.phys),
                                               state.contiguous().data_ptr(), self.grads.data_ptr(),
                                               self.flag.data_ptr(), out.data_ptr(), ct.byref(self.b.work.struct),
                                               _lib.stream_ptr()), "fvm_residual_state")
        return out


class CorrectorModel:
    """Network + the normalisation, geometry and residual baseline of one batch of meshes."""

    def __init__(self, batch, case_params: torch.Tensor, k: int = 8, seed: int = 0, lr: float = 1e-3,
                 like: "CorrectorModel | None" = None):
        """``like``: reuse another model's trained network and normalisation on this batch of meshes
        (the weights are mesh-independent; neighbours and geometry are this batch's)."""
        self.batch = batch
        self.k = k if like is None else like.k
        C = batch.n_comp
        self.C = C
        kt = batch.kt
        dev = batch.device
        self.net = CorrectorNet(C, device=dev, seed=seed, lr=lr) if like is None else like.net
        self.nbr = neighbour_table(kt).to(dev)
        self.cell_case = batch.dev.case["cell_case"].long().to(dev)
        cp = case_params[self.cell_case.cpu()]
        lengths = (2.0, 1.0) if kt.dim == 2 else (20.0, 10.0, 10.0)   # channel / sphere box extents
        self.geo = geometry_features(kt, cp, lengths).to(dev)
        if 2 * C + self.geo.shape[1] > XW:
            raise ValueError("too many input features")
        self.vol = kt.volumes.to(dev).double()
        self.case_vol = torch.zeros(batch.n_cases, dtype=torch.float64, device=dev).index_add_(
            0, self.cell_case, self.vol)
        self.cons = slice(batch.mesh.dim, batch.mesh.dim + 2)          # mass and energy components
        self.res = ResidualEval(batch)
        N = batch.n_cells
        self.cell_case32 = batch.dev.case["cell_case"]
        self.kdt_case = torch.empty(batch.n_cases, device=dev)
        self.S = torch.empty((batch.n_cases, C), dtype=torch.float64, device=dev)
        self.shift = torch.zeros((batch.n_cases, C), device=dev)
        self.base = torch.empty((N, C), device=dev)
        self.fmean = torch.zeros(2 * C, device=dev)
        self.finv = torch.ones(2 * C, device=dev)
        self.scale = torch.ones(C, device=dev)
        if like is not None:
            self.fmean, self.finv, self.scale = like.fmean, like.finv, like.scale

    def save(self, path: str, meta: dict | None = None):
        """Network weights, the input / output normalisation and k (mesh-independent: a model
        loaded onto another batch of meshes with ``load`` proposes the same way)."""
        torch.save({"net": self.net.state_dict(), "k": self.k, "fmean": self.fmean.cpu(), "finv": self.finv.cpu(),
                    "scale": self.scale.cpu(), "meta": meta or {}}, path)

    @classmethod
    def load(cls, path: str, batch, case_params: torch.Tensor) -> "CorrectorModel":
        d = torch.load(path, map_location="cpu", weights_only=True)
        m = cls(batch, case_params, k=int(d["k"]))
        m.net.load_state_dict(d["net"])
        dev = batch.device
        m.fmean, m.finv, m.scale = d["fmean"].to(dev), d["finv"].to(dev), d["scale"].to(dev)
        m.meta = d.get("meta", {})
        return m

    def kdt(self) -> torch.Tensor:
        """k * dt of each cell's case, [N][1] (read from the solver's device time steps)."""
        return (self.k * self.batch.t_solver.dt)[self.cell_case].unsqueeze(1)

    def set_normalisation(self, feats: torch.Tensor, targets: torch.Tensor):
        """feats [S][N][2C] = [U, base]; targets [S][N][C] = U_{t+k} - U_t - base.  In
        data-parallel training the first rank's statistics are used by every rank."""
        self.fmean = feats.mean(dim=(0, 1)).float().contiguous()
        self.finv = (1.0 / (feats.std(dim=(0, 1)) + 1e-12)).float().contiguous()
        self.scale = (targets.std(dim=(0, 1)) + 1e-12).float().contiguous()
        broadcast_from_first([self.fmean, self.finv, self.scale], self.net.bucket.group)

    def inputs(self, state: torch.Tensor, r0: torch.Tensor):
        """Writes base = k dt r0 and the network input features for (state, base); returns them."""
        b = self.net._alloc(state.shape[0])
        torch.mul(self.batch.t_solver.dt, float(self.k), out=self.kdt_case)
        _lib.check(self.net.lib.fvm_corrector_inputs(
            state.data_ptr(), r0.data_ptr(), self.kdt_case.data_ptr(), self.cell_case32.data_ptr(), state.shape[0],
            self.C, self.fmean.data_ptr(), self.finv.data_ptr(), self.geo.data_ptr(), self.geo.shape[1],
            self.base.data_ptr(), b["X"].data_ptr(), XW, _lib.stream_ptr()), "fvm_corrector_inputs")
        return b["X"]

    def _shift(self, out: torch.Tensor) -> torch.Tensor:
        """Per-case offsets that remove the volume-weighted mean of the mass and energy parts of
        scale * out (the other components get no offset)."""
        b = self.batch
        _lib.check(self.net.lib.fvm_conservation(ct.byref(b.dev.struct), out.data_ptr(), self.S.data_ptr(),
                                                 ct.byref(b.work.struct), _lib.stream_ptr()), "fvm_conservation")
        mean = self.S[:, self.cons] / self.case_vol.unsqueeze(1) * self.scale[self.cons].double()
        self.shift[:, self.cons] = mean.float()
        return self.shift

    def predict(self, state: torch.Tensor, out_state: torch.Tensor, r0: torch.Tensor):
        """out_state = proposal for U_{t+k} from state = U_t with residual r0 = dU/dt(U_t)."""
        self.inputs(state, r0)
        out = self.net.forward(self.nbr, store_pre=False)
        shift = self._shift(out)
        _lib.check(self.net.lib.fvm_corrector_combine(
            state.data_ptr(), self.base.data_ptr(), out.data_ptr(), self.scale.data_ptr(), shift.data_ptr(),
            self.cell_case32.data_ptr(), state.shape[0], self.C, out_state.data_ptr(), _lib.stream_ptr()),
            "fvm_corrector_combine")
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


def train(model: CorrectorModel, traj: torch.Tensor, iters: int, seed: int = 0, log_every: int = 0,
          normalise: bool = True) -> list:
    """Adam on random windows (U_t -> U_{t+k}) of a recorded trajectory; returns the loss history.
    ``normalise``: first set the input / output normalisation from this trajectory (off when the
    model continues training on a new batch of meshes)."""
    k = model.k
    T = traj.shape[0] - k
    r0 = torch.empty_like(traj[0])
    if normalise:
        feats, tg = [], []
        for t in range(0, T, max(1, T // 40)):
            model.res(traj[t], r0)
            base = model.kdt() * r0
            feats.append(torch.cat([traj[t], base], 1))
            tg.append(traj[t + k] - traj[t] - base)
        model.set_normalisation(torch.stack(feats), torch.stack(tg))
        del feats, tg
    g = torch.Generator().manual_seed(seed)
    target = torch.empty_like(traj[0])
    losses = []
    model.net._alloc(traj.shape[1])
    for it in range(iters):
        t = int(torch.randint(0, T, (1,), generator=g))
        model.res(traj[t], r0)
        model.inputs(traj[t], r0)
        torch.sub(traj[t + k], traj[t], out=target)
        target.sub_(model.base).div_(model.scale)
        loss = model.net.train_step(model.nbr, target)
        if log_every and (it % log_every == 0 or it == iters - 1):
            losses.append((it, float(loss.item())))
    model.net.check_errors()
    return losses


def train_streaming(make_batch, n_batches: int, iters: int, k: int = 8, record: int = 100, spinup: int = 200,
                    seed: int = 0, lr: float = 1e-3, prefetch=None, log=None, keep: dict | None = None,
                    group=None) -> tuple:
    """Train one network on a stream of mesh batches (many more cases than fit on the device).

    ``make_batch(b)`` -> (BatchedFVM with its time steps set, case parameters [cases][2]) builds
    batch b; ``prefetch(b)`` (optional) starts building batch b ahead of time.  Each batch is
    spun up ``spinup`` steps and ``record`` + k steps are recorded; ``iters / n_batches`` Adam
    iterations then draw random windows from it.  The normalisation comes from the first batch,
    and the network and the Adam moments carry over.  ``keep`` (a dict), when given, holds the
    current model under "model" after each batch (for periodic saving by ``log``).  ``group``:
    data-parallel training over its ranks (each rank streams its own batches, all ranks take the
    same number of batches and iterations; gradients are averaged every iteration).  Returns
    (model, loss history, cases seen)."""
    model, hist, cases = None, [], 0
    per = max(1, iters // n_batches)
    done = 0
    for b in range(n_batches):
        if prefetch is not None and b + 1 < n_batches:
            prefetch(b + 1)
        batch, prm = make_batch(b)
        traj = record_trajectory(batch, steps=record + k, spinup=spinup)
        if model is None:
            m = CorrectorModel(batch, prm, k=k, seed=seed, lr=lr)
            m.net.data_parallel(group)
        else:
            m = CorrectorModel(batch, prm, like=model)
        n_it = per if b < n_batches - 1 else max(per, iters - done)
        h = train(m, traj, iters=n_it, seed=seed + b, log_every=max(1, n_it // 2), normalise=model is None)
        hist.extend((done + it, loss) for it, loss in h)
        done += n_it
        cases += batch.n_cases
        model = m
        if keep is not None:
            keep["model"] = model
        del traj
        if log is not None:
            log(b, done, cases, h[-1][1])
    return model, hist, cases


class CheckedRollout:
    """Corrector + fallback rollout on a batch, with per-case acceptance checks (see module doc)."""

    def __init__(self, model: CorrectorModel, drift_tol: float = 1e-4, residual_ratio: float = 3.0,
                 use_graphs: bool = True, consistency: float | None = None):
        self.m = model
        b = model.batch
        self.b = b
        self.lib = _lib.load()
        self.drift_tol, self.ratio = drift_tol, residual_ratio
        self.consistency = consistency or 0.0
        N, C = b.cells.state.shape
        d = b.device
        self.prop = torch.empty((N, C), device=d)
        self.r0 = torch.empty((N, C), device=d)
        self.r1 = torch.empty((N, C), device=d)
        self.vol32 = model.vol.float().contiguous()
        self.check_sums = torch.zeros((b.n_cases, 3 * C + 4), dtype=torch.float64, device=d)
        self.ok_u8 = torch.zeros(b.n_cases, dtype=torch.uint8, device=d)
        self.ok = self.ok_u8.view(torch.bool)
        self.use_graphs = use_graphs
        self._g_propose = None
        self._fallback = None
        b.use_case_mask(True)             # the fallback advances only the cases that failed
        self.accepted = 0
        self.windows = 0
        self.full_windows = 0

    def _propose(self):
        """Proposal and its checks; leaves the per-case verdicts in ``self.ok`` (device).

        ``fvm_corrector_checks`` reduces, per case and in FP64, the volume-weighted sums of the state,
        the proposal and r0 (conservation: the proposal's mass and energy must equal the state's plus
        k dt times r0's, to ``drift_tol`` relative), the squared residual norms of state and proposal
        (|r1|^2 <= ratio^2 |r0|^2), the number of inadmissible proposal cells (density or internal
        energy <= 0, or not finite) and, with ``consistency``, the proposal's distance to the
        trapezoidal rule over the window (|U' - U - k dt (r0 + r1) / 2| <= consistency k dt |r0|),
        then writes the verdicts: two launches after the proposal."""
        b, k = self.b, self.m.k
        U = b.cells.state
        self.m.res(U, self.r0)
        self.m.predict(U, self.prop, self.r0)
        self.m.res(self.prop, self.r1)
        N, C = U.shape
        _lib.check(self.lib.fvm_corrector_checks(
            U.data_ptr(), self.prop.data_ptr(), self.r0.data_ptr(), self.r1.data_ptr(), self.vol32.data_ptr(),
            self.m.cell_case32.data_ptr(), N, C, b.n_cases, b.t_solver.dt.data_ptr(), k, float(self.drift_tol),
            float(self.ratio), float(self.consistency), self.check_sums.data_ptr(), self.ok_u8.data_ptr(), None,
            _lib.stream_ptr()),
            "fvm_corrector_checks")

    def _run_propose(self):
        if not self.use_graphs:
            self._propose()
            return
        if self._g_propose is None:
            self._propose()                                  # eager once: allocates the network buffers
            s = torch.cuda.Stream(device=self.b.device)
            s.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    self._propose()
            torch.cuda.current_stream().wait_stream(s)
            self._g_propose = g
        self._g_propose.replay()

    def _run_fallback(self):
        sol, k = self.b.t_solver, self.m.k
        if not self.use_graphs:
            sol.step(k)
            return
        sol._sync_prims()
        if self._fallback is None:
            self._fallback = sol.graph_steps(k)
        self._fallback()

    def window(self) -> torch.Tensor:
        """Advance one window of k steps; returns the per-case acceptance mask (host)."""
        b = self.b
        self._run_propose()
        ok = self.ok.cpu()
        self.windows += b.n_cases
        if bool(ok.all()):
            b.cells.state = self.prop
            self.accepted += b.n_cases
            self.full_windows += 1
            return ok
        # fallback: k plain FVM steps for the cases that failed (the others are frozen), then the
        # accepted proposals replace the frozen cases' states
        keep = self.ok[self.m.cell_case].unsqueeze(1)
        b.active.copy_(~self.ok)
        self._run_fallback()
        b.active.fill_(1)
        b.cells.state = torch.where(keep, self.prop, b.cells.state)
        self.accepted += int(ok.sum())
        return ok
