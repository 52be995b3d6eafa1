"""Corrector network: hand-written forward/backward vs torch autograd, training, checked rollout.

The torch reference rounds to bf16 exactly where the CUDA path does (GEMM operands: features,
the fp32 activations and their neighbour mean, weights) and accumulates in fp32, so forward outputs agree to ~1e-3 relative and
weight gradients to ~1e-2 relative (bf16 rounding of the backward operands dZ and A).
Needs a B200.
"""
import copy

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    from fvm_solver_b200 import batched as B, workloads as W
    cases, params = [], []
    for i, n in enumerate([2100, 3300, 2600]):
        p = W.ensemble_params(i)
        p["n_cells"] = n
        c = W.channel_cylinder(device="cuda", solver_name="Butcher", solver_extra="SSP_RK3", **p)
        c.cfg.cfl = None
        cases.append(c)
        params.append([p["mach"], np.log10(p["reynolds"])])
    parts = [B.build_case_tables(c) for c in cases]
    batch = B.BatchedFVM(parts, cases[0].cfg, device="cuda")
    batch.t_solver.update_cfl_dt(0.5)
    return batch, torch.tensor(params, dtype=torch.float32)


def _torch_reference(net, X, nbr, target, N):
    """The network in torch with the CUDA path's bf16 rounding points; returns out, loss, grads."""
    bf = lambda t: t.to(torch.bfloat16).float()
    P = {k: v.detach().clone().requires_grad_(True) for k, v in net.params.items()}
    x = X[:N].float()
    z = x @ bf(P["W_in"]).t() + P["b_in"]
    h = torch.nn.functional.silu(z)
    nb = nbr.long()
    valid = (nb >= 0)
    for l in range(net.L):
        # the neighbour mean of the fp32 stream, then both halves of the GEMM operand in bf16
        gathered = torch.where(valid.unsqueeze(-1), h[nb.clamp(min=0)], torch.zeros(()).cuda())
        mean = gathered.sum(1) / valid.sum(1, keepdim=True).clamp(min=1)
        A = torch.cat([bf(h), bf(mean)], 1)
        z = A @ bf(P[f"W{l}"]).t() + P[f"b{l}"]
        h = h + torch.nn.functional.silu(z)
    out = h @ P["W_out"].t() + P["b_out"]
    loss = ((out - target) ** 2).mean()
    loss.backward()
    return out.detach(), loss.detach(), {k: v.grad for k, v in P.items()}


def test_forward_backward_vs_autograd(small_batch):
    from fvm_solver_b200.corrector import CorrectorModel
    batch, params = small_batch
    model = CorrectorModel(batch, params, seed=3, lr=0.0)          # lr 0: the step leaves weights unchanged
    U = batch.cells.state.clone()
    r0 = model.res(U, torch.empty_like(U))
    model.set_normalisation(torch.cat([U, U * 1e-3], 1).unsqueeze(0), (U * 1e-3 + 1e-3).unsqueeze(0))
    N = U.shape[0]
    X = model.inputs(U, r0).clone()
    target = torch.randn(N, 4, device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
    ref_out, ref_loss, ref_g = _torch_reference(model.net, X, model.nbr, target, N)
    out = model.net.forward(model.nbr).clone()
    assert rel_l2(out.cpu().numpy(), ref_out.cpu().numpy()) < 2e-3
    # inference runs one persistent fused kernel per layer (neighbour mean in shared memory, the
    # decoder in the last layer's epilogue): bitwise the same output
    assert torch.equal(model.net.forward(model.nbr, store_pre=False), out)
    grads_before = {k: v.clone() for k, v in model.net.grads.items()}
    assert all(float(v.abs().max()) == 0.0 for v in grads_before.values())
    # capture the gradients: run the backward pass but stop Adam from zeroing them
    net = model.net
    saved_adam = net.adam
    net.adam = lambda *a, **k: None
    loss = net.train_step(model.nbr, target)
    net.adam = saved_adam
    assert abs(float(loss.item()) / float(ref_loss) - 1) < 2e-3
    for k in ref_g:
        assert rel_l2(net.grads[k].cpu().numpy(), ref_g[k].cpu().numpy()) < 3e-2, k
    net.check_errors()


def test_training_reduces_loss_and_rollout(small_batch):
    from fvm_solver_b200.corrector import CheckedRollout, CorrectorModel, record_trajectory, train
    batch, params = small_batch
    traj = record_trajectory(batch, steps=60, spinup=10)
    model = CorrectorModel(batch, params, k=8, seed=1, lr=2e-3)
    hist = train(model, traj, iters=300, log_every=50)
    assert hist[-1][1] < 0.5 * hist[0][1]
    # the proposal changes each case's mass and energy by exactly k dt sum(vol dU/dt)
    U = batch.cells.state.clone()
    r0 = model.res(U, torch.empty_like(U))
    prop = model.predict(U, torch.empty_like(U), r0)
    vol = model.vol.unsqueeze(1)
    cc = model.cell_case
    dM = torch.zeros(batch.n_cases, 4, dtype=torch.float64, device="cuda").index_add_(0, cc, (prop - U).double() * vol)
    want = torch.zeros_like(dM).index_add_(0, cc, r0.double() * vol) * (model.k * batch.t_solver.dt.double())[:, None]
    M = torch.zeros_like(dM).index_add_(0, cc, U.double() * vol)
    assert float(((dM - want)[:, 2:].abs() / M[:, 2:].abs()).max()) < 1e-5
    # graph-replayed and eager rollouts agree
    start = batch.cells.state.clone()
    g_start, f_start = batch.grads.clone(), batch.has_grads.clone()
    ro = CheckedRollout(model)
    oks = []
    for _ in range(3):
        ok = ro.window()
        assert ok.shape == (batch.n_cases,)
        oks.append(ok)
    assert torch.isfinite(batch.cells.state).all()
    assert 0 <= ro.accepted <= ro.windows
    end_graph = batch.cells.state.clone()
    batch.cells.state = start
    batch.grads.copy_(g_start)
    batch.has_grads.copy_(f_start)
    ro2 = CheckedRollout(model, use_graphs=False)
    for w in range(3):
        ok = ro2.window()
        assert torch.equal(ok, oks[w])
    rel = float((batch.cells.state - end_graph).norm() / end_graph.norm())
    assert rel < 1e-5


def test_corrector_3d_sphere_batch():
    """The corrector on a batch of two small 3D sphere cases (C = 5): training lowers the loss, the
    proposal keeps each case's mass and energy change at k dt sum(vol dU/dt), rollouts stay finite."""
    import copy
    import numpy as np
    from fvm_solver_b200 import batched as B, workloads as W
    from fvm_solver_b200.corrector import CheckedRollout, CorrectorModel, record_trajectory, train
    parts = B.build_ensemble_tables(2, base_seed=77, family="sphere", cells=(15_000, 25_000))
    cfg = copy.deepcopy(W.sphere_case(0, device="cuda", base_seed=77, cells=(15_000, 15_000)).cfg)
    cfg.solver_name, cfg.solver_extra, cfg.cfl = "Butcher", "SSP_RK3", None
    prm = torch.tensor([[W.sphere_params(i, 77)["mach"], np.log10(W.sphere_params(i, 77)["reynolds"])]
                        for i in range(2)], dtype=torch.float32)
    batch = B.BatchedFVM(parts, cfg, device="cuda")
    batch.t_solver.update_cfl_dt(0.5)
    traj = record_trajectory(batch, steps=40, spinup=5)
    model = CorrectorModel(batch, prm, k=8, seed=2, lr=2e-3)
    hist = train(model, traj, iters=200, log_every=50)
    assert hist[-1][1] < hist[0][1]
    U = batch.cells.state.clone()
    r0 = model.res(U, torch.empty_like(U))
    prop = model.predict(U, torch.empty_like(U), r0)
    vol = model.vol.unsqueeze(1)
    cc = model.cell_case
    dM = torch.zeros(2, 5, dtype=torch.float64, device="cuda").index_add_(0, cc, (prop - U).double() * vol)
    want = torch.zeros_like(dM).index_add_(0, cc, r0.double() * vol) * (model.k * batch.t_solver.dt.double())[:, None]
    M = torch.zeros_like(dM).index_add_(0, cc, U.double() * vol)
    assert float(((dM - want)[:, 3:].abs() / M[:, 3:].abs()).max()) < 1e-5
    ro = CheckedRollout(model)
    for _ in range(2):
        assert ro.window().shape == (2,)
    assert torch.isfinite(batch.cells.state).all()


@pytest.mark.parametrize("N,KN", [(1000, 4), (77, 3), (300_001, 4)])
def test_fused_layer_matches_separate_kernels(N, KN):
    """fvm_mp_layer (persistent: loader warps, tcgen05 MMA, epilogue warps, two stages) against
    fvm_mp_gather_f32 + fvm_gemm_bf16 + fvm_decoder_f32: bitwise, on a ragged last tile, a single
    partial tile and enough tiles that every CTA cycles its stages and accumulators many times."""
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    from fvm_solver_b200 import _lib
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(N + KN)
    h = torch.randn(N, 64, device="cuda", generator=g)
    nbr = torch.randint(-1, N, (N, KN), device="cuda", generator=g, dtype=torch.int32)
    Wt = (0.1 * torch.randn(64, 128, device="cuda", generator=g)).to(torch.bfloat16).contiguous()
    bias = torch.randn(64, device="cuda", generator=g)
    Wo = torch.randn(5, 64, device="cuda", generator=g)
    bo = torch.randn(5, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = _lib.stream_ptr()
    # separate kernels
    A = torch.empty(N, 128, dtype=torch.bfloat16, device="cuda")
    _lib.check(lib.fvm_mp_gather_f32(h.data_ptr(), nbr.data_ptr(), N, KN, A.data_ptr(), s), "gather")
    want = torch.empty(N, 64, device="cuda")
    _lib.check(lib.fvm_gemm_bf16(A.data_ptr(), 128, Wt.data_ptr(), 128, N, 64, 128, 1, bias.data_ptr(), h.data_ptr(),
                                 64, want.data_ptr(), None, 64, None, 1, err.data_ptr(), s), "gemm")
    want_out = torch.empty(N, 5, device="cuda")
    _lib.check(lib.fvm_decoder_f32(want.data_ptr(), Wo.data_ptr(), bo.data_ptr(), N, 5, want_out.data_ptr(), s), "dec")
    # fused layer: h_out, then the decoder form
    got = torch.full((N, 64), float("nan"), device="cuda")
    _lib.check(lib.fvm_mp_layer(h.data_ptr(), nbr.data_ptr(), N, KN, Wt.data_ptr(), bias.data_ptr(), got.data_ptr(),
                                None, None, 5, None, err.data_ptr(), s), "layer")
    got_out = torch.full((N, 5), float("nan"), device="cuda")
    _lib.check(lib.fvm_mp_layer(h.data_ptr(), nbr.data_ptr(), N, KN, Wt.data_ptr(), bias.data_ptr(), None,
                                Wo.data_ptr(), bo.data_ptr(), 5, got_out.data_ptr(), err.data_ptr(), s), "layer+dec")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(got, want)
    assert torch.equal(got_out, want_out)
    # and against torch (bf16 operands, fp32 accumulation)
    hv = h.double()
    valid = nbr >= 0
    nb = nbr.long().clamp(min=0)
    mean = (torch.where(valid.unsqueeze(-1), h[nb], torch.zeros((), device="cuda")).sum(1)
            * (1.0 / valid.sum(1, keepdim=True).clamp(min=1).float()))
    Aref = torch.cat([h.to(torch.bfloat16), mean.to(torch.bfloat16)], 1).double()
    ref = hv + torch.nn.functional.silu(Aref @ Wt.double().t() + bias.double())
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < 1e-5


def _checks_torch(U, P, r0, r1, vol, cc, n, dt, k, tol, ratio, dim, consistency=0.0):
    """The acceptance checks written as torch reductions (FP64 sums of FP32 products)."""
    def sums(x):
        return torch.zeros((n, x.shape[1]), dtype=torch.float64, device=x.device).index_add_(
            0, cc, x.double() * vol.double()[:, None])
    M0, Mp, R0 = sums(U), sums(P), sums(r0)
    cons = slice(dim, dim + 2)
    drift = ((Mp[:, cons] - (M0[:, cons] + k * dt.double()[:, None] * R0[:, cons])).abs()
             / M0[:, cons].abs()).max(dim=1).values
    n0, n1 = sums(r0 * r0).sum(dim=1), sums(r1 * r1).sum(dim=1)
    rho = P[:, dim]
    e_int = P[:, dim + 1] - 0.5 * P[:, :dim].square().sum(dim=1) / rho
    bad = torch.zeros(n, dtype=torch.float64, device=U.device).index_add_(
        0, cc, ((rho <= 0) | (e_int <= 0) | ~torch.isfinite(e_int)).double())
    kdt = k * dt.double()
    e = (P.double() - U.double()) - 0.5 * kdt[cc, None] * (r0.double() + r1.double())
    e2 = torch.zeros(n, dtype=torch.float64, device=U.device).index_add_(0, cc, (e * e).sum(dim=1) * vol.double())
    ok = (drift <= tol) & (n1 <= ratio ** 2 * n0) & torch.isfinite(drift) & (bad == 0)
    if consistency > 0:
        ok &= e2 <= consistency ** 2 * kdt ** 2 * n0
    return ok, M0, Mp, R0, n0, n1, bad, e2


@pytest.mark.parametrize("C", [4, 5])
def test_checks_kernel_matches_torch(C):
    """fvm_corrector_checks against the torch reductions, with failures of each kind planted in
    their own cases, with and without the trapezoid gate, each twice in a row (the kernel leaves its
    sums buffer zeroed)."""
    if not torch.cuda.is_available():
        pytest.skip("needs CUDA")
    from fvm_solver_b200 import _lib
    lib = _lib.load()
    g = torch.Generator().manual_seed(C)
    dim, n, k, tol, ratio = C - 2, 41, 8, 1e-4, 3.0
    sizes = torch.randint(1, 9000, (n,), generator=g)
    cc = torch.repeat_interleave(torch.arange(n), sizes).cuda()
    N = int(sizes.sum())
    vol = (0.5 + torch.rand(N, generator=g)).cuda()
    U = torch.rand((N, C), generator=g).cuda()
    U[:, dim] += 1.0                                     # density
    U[:, dim + 1] += 3.0                                 # energy above the kinetic part
    r0 = (torch.rand((N, C), generator=g) - 0.5).cuda()
    dt = (1e-4 * (1 + torch.rand(n, generator=g))).cuda()
    kdt = k * dt[cc, None]
    P = U + kdt * r0
    r1 = 0.5 * r0                                        # trapezoid distance 0.25 k dt |r0|
    first = torch.cumsum(sizes, 0) - sizes
    P[int(first[1]), dim] = -1.0                          # case 1: negative density in one cell
    P[cc == 2, dim + 1] *= 1.01                          # case 2: energy drift
    r1[cc == 3] = 4.0 * r0[cc == 3]                       # case 3: residual grew beyond the ratio
    P[int(first[4]) + int(sizes[4]) - 1, 0] = float("nan")  # case 4: non-finite proposal
    P[cc == 5, dim] *= 1.00001                           # case 5: mass drift 1e-5, inside the tolerance
    m6 = cc == 6                                         # case 6: trapezoid distance 0.75 k dt |r0|
    P[m6] += 0.5 * kdt[m6] * r0[m6]
    sums = torch.zeros((n, 3 * C + 4), dtype=torch.float64, device="cuda")
    keep = torch.empty_like(sums)
    cc32 = cc.int()
    scale = sizes.double().cuda()                        # bound on each sum's absolute terms (order 1 each)
    for consistency in (0.0, 0.3):
        want, M0, Mp, R0, n0, n1, bad, e2 = _checks_torch(U, P, r0, r1, vol, cc, n, dt, k, tol, ratio, dim,
                                                          consistency)
        assert want[[0, 5]].all() and not want[[1, 2, 3, 4]].any()
        assert bool(want[6]) == (consistency == 0.0)
        for _ in range(2):
            ok = torch.zeros(n, dtype=torch.uint8, device="cuda")
            _lib.check(lib.fvm_corrector_checks(U.data_ptr(), P.data_ptr(), r0.data_ptr(), r1.data_ptr(),
                                                vol.data_ptr(), cc32.data_ptr(), N, C, n, dt.data_ptr(), k, tol, ratio,
                                                consistency, sums.data_ptr(), ok.data_ptr(), keep.data_ptr(),
                                                _lib.stream_ptr()), "fvm_corrector_checks")
            torch.cuda.synchronize()
            assert torch.equal(ok.bool(), want)
            assert float(sums.abs().max()) == 0.0
            for got, ref in ((keep[:, :C], M0), (keep[:, 2 * C:3 * C], R0), (keep[:, 3 * C], n0),
                             (keep[:, 3 * C + 1], n1)):
                sc = scale if got.dim() == 1 else scale[:, None]
                assert float(((got - ref).abs() / sc).max()) < 1e-13
            finite = torch.isfinite(Mp).all(dim=1)
            assert float(((keep[finite, C:2 * C] - Mp[finite]).abs() / scale[finite, None]).max()) < 1e-13
            assert torch.equal(keep[:, 3 * C + 2], bad)
            fin = torch.isfinite(e2)
            assert float(((keep[fin, 3 * C + 3] - e2[fin]).abs() / (e2[fin] + 1e-30)).max()) < 1e-9
