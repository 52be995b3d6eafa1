"""CPU oracle: numpy restatement of the reference's residual and time integrators.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path; only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs use it.  The product
(``fvm_solver_b200``) never imports it.

It restates, step by step, the reference's FP32 PyTorch path (``compile=False``):

* ELL SpMV/SpMM                       ``time_fvm/utils/ell_kernel.py:25-80, 100-173``
* boundary face values                ``time_fvm/fvm_stepping/facet_boundary.py:124-168``
* characteristic BC                   ``time_fvm/fvm_stepping/facet_boundary.py:418-512``
* LSQ cell gradients                  ``time_fvm/fvm_stepping/facet_process.py:409-418``
* limited face values                 ``time_fvm/fvm_stepping/facet_process.py:387-407``,
                                      ``time_fvm/fvm_stepping/limiter.py:29-87``
* facet assembly, face gradients      ``time_fvm/fvm_stepping/facet_process.py:332-385, 420-450``
* stress / EOS                        ``time_fvm/fvm_equation.py:62-187``
* facet fluxes and divergence         ``time_fvm/fvm_equation.py:199-435``
* state <-> primitive conversion      ``time_fvm/fvm_equation.py:35-55``
* Butcher / adaptive / SSP integrators ``time_fvm/time_solvers/integrators.py:42-393``
* Adams-Bashforth 3 (restated; the reference's Adams3PC cannot run), CFL time step (new).

Input is an ``fvm_solver_b200.tables.FVMTables`` instance: its reference-format operators and
mesh arrays are bit-identical to what the reference assembles (pinned by the golden fixtures),
so the oracle sees exactly the reference's operands.  ``dtype`` selects float32 (parity with the
reference's FP32 path) or float64.

Parity pinning: the oracle is checked against golden vectors produced by running the reference
itself (``tests/golden/make_golden.py``) -- residuals, limited gradients and integrator steps on a
2D channel-cylinder mesh and a 3D box mesh, in FP32 and FP64, and the first residual and ten
SSP-RK3 steps on two larger meshes (the 11 307-triangle channel mesh of the channel-cylinder
benchmark, a 9 066-tet box).
"""
from __future__ import annotations

import numpy as np

# ---------------------------------------------------------------------------------------------
# Sparse operators (ell_kernel.py): y = A x (+ b), A in row-major ELL.
# ---------------------------------------------------------------------------------------------


def ell_from_coo(A, dtype=np.float32):
    """Row-major ELL (vals [M, K], cols [M, K]) of a torch COO matrix, ascending columns per row."""
    from fvm_solver_b200.tables import coo_to_ell   # host packing, bit-identical to csr_to_ell
    v, c = coo_to_ell(A)
    return v.numpy().astype(dtype), c.numpy().astype(np.int64)


def ell_spmv(vals, cols, x, b=None):
    """``ell_spmv`` (ell_kernel.py:135-173): accumulate slot by slot, then add the bias."""
    acc = np.zeros(vals.shape[0], dtype=vals.dtype)
    for k in range(vals.shape[1]):
        acc = acc + vals[:, k] * x[cols[:, k]]
    if b is not None:
        acc = acc + b
    return acc


def ell_spmm(vals, cols, X, b=None):
    """``ell_spmm`` (ell_kernel.py:176-210): Y[M, B] = A X (+ b[:, None])."""
    acc = np.zeros((vals.shape[0], X.shape[1]), dtype=vals.dtype)
    for k in range(vals.shape[1]):
        acc = acc + vals[:, k, None] * X[cols[:, k]]
    if b is not None:
        acc = acc + b[:, None]
    return acc


# ---------------------------------------------------------------------------------------------
# Slope limiters (limiter.py:29-77)
# ---------------------------------------------------------------------------------------------
def limiter_phi(p, delta, dU, eps):
    if p == 1:
        s = 2 * ((dU > 0).astype(dU.dtype) - 0.5) * (np.abs(dU) + 1e-8)
        return np.clip(delta / s, 0.0, 1.0)
    if p == 2:
        return (delta ** 2 + eps + 2 * delta * dU) / (delta ** 2 + 2 * dU ** 2 + delta * dU + eps)
    a, b = np.abs(delta), np.abs(dU)
    with np.errstate(divide="ignore", invalid="ignore"):
        if p == 3:
            a_eps = a ** 3 + eps
            S = 4 * b ** 2
            phi = (a_eps + a * S) / (a_eps + b * (delta ** 2 + S))
            return np.where(a < 2 * b, phi, 1)
        if p == 4:
            b2 = 2 * b
            a_eps = a ** 4 + eps
            S = b2 * (a * a + b2 * (b2 - a))
            phi = (a_eps + a * S) / (a_eps + b * (delta ** 3 + S))
            return np.where(a < b2, phi, 1)
        if p == 5:
            a_eps = a ** 5 + eps
            S = 8 * b ** 2 * (a ** 2 - 2 * b * (a - b))
            phi = (a_eps + a * S) / (a_eps + b * (delta ** 4 + S))
            return np.where(a < 2 * b, phi, 1)
    raise NotImplementedError(f"Limiter of order {p} is not implemented.")


# ---------------------------------------------------------------------------------------------
# Residual
# ---------------------------------------------------------------------------------------------
class OracleResidual:
    """``FVMEquation.forward`` restated (fvm_equation.py:406-435) on one mesh."""

    def __init__(self, tables, cfg, dtype=np.float32):
        t = tables
        f = lambda a: a.detach().cpu().numpy().astype(dtype)
        i = lambda a: a.detach().cpu().numpy().astype(np.int64)
        self.dt = dtype
        self.dim, self.C = t.dim, t.n_comp
        self.N, self.F, self.Fb = t.n_cells, t.n_facets, t.n_bc
        self.K = t.dim + 1
        # physics constants (fvm_equation.py:23-33)
        self.T_0, self.mu, self.mu_b = cfg.T_0, cfg.viscosity, cfg.visc_bulk
        self.S, self.C_v, self.gamma = cfg.S_const, cfg.C_v, cfg.gamma
        self.R = cfg.C_v * (cfg.gamma - 1)
        self.kappa, self.v_factor, self.lim_p = cfg.thermal_cond, cfg.v_factor, cfg.lim_p
        ops = t.ops
        self.G = ell_from_coo(ops.G_mats, dtype)
        self.Fm = ell_from_coo(ops.flux_mat, dtype)
        self.Afg = ell_from_coo(ops.A_face_grad, dtype)
        self.b_fg = f(ops.b_face_grad)
        if self.Fb:
            self.Abc = ell_from_coo(ops.A_bc, dtype)
            self.b_bc = f(ops.b_bc)
            self.Acorr = ell_from_coo(ops.A_corr, dtype)
        self.neigh = i(t.neigh_combine)
        self.disp = f(t.cent_to_facet_disp.squeeze(-1))        # [N, K, dim]
        self.eps = f(t.eps_p)                                  # [N, 1, 1]
        self.c2f = i(t.cell_to_facet)
        self.signs = i(t.cell_facet_signs)
        self.bc_loc = i(t.bc_locations)
        self.bc_side = i(t.bc_facet_side)
        self.f2c_bc = i(t.facet_to_cell_bc)
        self.normals = f(t.normals)
        self.fsize = f(t.facet_size)                           # [F, 1]
        self.nhat = f(t.normals_hat.squeeze(-1))               # [F, dim]
        self.xorth = f(t.X_orthog)                             # [F, dim]
        self.groups = []
        for g in t.char_groups.values():
            self.groups.append(dict(bc_idx=i(g.bc_idx), cells=i(g.cells), n=f(g.normals),
                                    rho=f(g.rho_inf), vn=f(g.v_n_inf), vt=f(g.v_t_inf), p=f(g.p_inf)))
        self.grad_comps = list(range(self.dim)) + [self.dim + 1]

    # -- EOS (fvm_equation.py:73-83) --
    def eos_c(self, T):
        return np.sqrt(self.gamma * self.R * T)

    def eos_P(self, rho, T):
        return self.R * rho * T

    # -- characteristic BC (facet_boundary.py:418-512) --
    def _bc_characteristic(self, U_face, Ucells, g):
        d = self.dim
        Vs, rho, T = Ucells[:, :d], Ucells[:, d], Ucells[:, d + 1]
        n = g["n"]
        vn = (Vs * n).sum(axis=1)
        vt = Vs - vn[:, None] * n
        p, c = self.eos_P(rho, T), self.eos_c(T)
        drho, dvn, dp = g["rho"] - rho, g["vn"] - vn, g["p"] - p
        inv_c = 1 / c
        inv_c2 = inv_c ** 2
        h_dp = 0.5 * inv_c2 * dp
        h_dvn = 0.5 * rho * inv_c * dvn
        x0, x1, x2 = -h_dvn + h_dp, drho - inv_c2 * dp, h_dvn + h_dp
        scale = 10.0 / c.mean(dtype=c.dtype)
        g0 = 0.5 * (1.0 - np.tanh(scale * (vn - c)))
        g1 = 0.5 * (1.0 - np.tanh(scale * vn))
        g2 = 0.5 * (1.0 - np.tanh(scale * (vn + c)))
        x0, x1, x2 = g0 * x0, g1 * x1, g2 * x2
        vtb = g1[:, None] * vt + (1.0 - g1[:, None]) * g["vt"]
        c2, cor = c * c, c / rho
        rho_b = rho + (x0 + x1 + x2)
        vn_b = vn + (-cor * x0 + cor * x2)
        p_b = p + c2 * (x0 + x2)
        V = vn_b[:, None] * n + vtb
        T_b = p_b / (self.R * rho_b)
        U_face[g["bc_idx"]] = np.concatenate([V, rho_b[:, None], T_b[:, None]], axis=1)

    def boundary_values(self, U, grads_prev):
        """``BoundarySetter.set_face_values`` (facet_boundary.py:124-145)."""
        C = self.C
        Uf = ell_spmv(*self.Abc, U.reshape(-1), self.b_bc)
        if grads_prev is not None:
            Uf = Uf + ell_spmv(*self.Acorr, grads_prev.reshape(-1))
        Uf = Uf.reshape(self.Fb, C)
        for g in self.groups:
            self._bc_characteristic(Uf, U[g["cells"]], g)
        return Uf

    def forward(self, U, grads_prev=None, return_faces=False):
        """Returns (dU/dt [N, C] in conserved variables, limited cell gradients [N, dim, C]); with
        ``return_faces`` also the facet values of both sides [F, 2, C] (``U_face_all``)."""
        U = np.asarray(U, dtype=self.dt)
        d, C, N, F, K = self.dim, self.C, self.N, self.F, self.K
        # 1-2. boundary facet values; cell + boundary value table
        Ub = self.boundary_values(U, grads_prev) if self.Fb else np.zeros((0, C), self.dt)
        Ucf = np.concatenate([U, Ub], axis=0)
        # 3. LSQ gradients (facet_process.py:409-418)
        grads = ell_spmm(*self.G, Ucf).reshape(N, d, C)
        # 4. limited face values (facet_process.py:387-407)
        Uc = U[:, None, :]
        Un = Ucf[self.neigh]
        dU = (grads[:, None, :, :] * self.disp[:, :, :, None]).sum(axis=2)
        Ucn = np.concatenate([Uc, Un], axis=1)
        up = Ucn.max(axis=1, keepdims=True) - Uc
        lo = Ucn.min(axis=1, keepdims=True) - Uc
        num = np.where(dU > 0, up, lo)
        phi = limiter_phi(self.lim_p, num, dU, self.eps).astype(self.dt)
        phi = phi.min(axis=1, keepdims=True)
        Us_face = (Uc + dU * phi).reshape(K * N, C)
        grads = grads * phi
        # 5. facet assembly (facet_process.py:349-351)
        Ufa = np.empty((F, 2, C), self.dt)
        Ufa[self.c2f, self.signs] = Us_face
        if self.Fb:
            Ufa[self.bc_loc, self.bc_side] = Ub
        Vs, rho, T = Ufa[:, :, :d], Ufa[:, :, d:d + 1], Ufa[:, :, d + 1:d + 2]
        mom = Vs * rho
        Q = rho * (self.C_v * T + 0.5 * (Vs ** 2).sum(axis=-1, keepdims=True))
        phi_n = (Vs * self.normals[:, None, :]).sum(axis=-1)
        # 7. facet gradients of (V, T) averaged over both sides (facet_process.py:362-371)
        gF = grads[:, :, self.grad_comps].reshape(N, d * (d + 1))
        gfa = np.empty((F, 2, d * (d + 1)), self.dt)
        gfa[self.c2f, self.signs] = np.repeat(gF, K, axis=0)
        if self.Fb:
            gfa[self.bc_loc, self.bc_side] = gF[self.f2c_bc]
        gls = ((gfa[:, 0] + gfa[:, 1]) / 2).reshape(F, d, d + 1)
        # 8-9. normal gradient + non-orthogonal correction (facet_process.py:374-385)
        gn = ell_spmv(*self.Afg, U.reshape(-1), self.b_fg).reshape(F, C)[:, self.grad_comps]
        dFdn = gn - (gls * self.xorth[:, :, None]).sum(axis=1)
        gdn = (gls * self.nhat[:, :, None]).sum(axis=1, keepdims=True)
        gFc = gls + (dFdn[:, None, :] - gdn) * self.nhat[:, :, None]
        grad_V = gFc[:, :, :d]
        grad_T_n = dFdn[:, -1]
        # stress (fvm_equation.py:101-120 / 149-170)
        Tm = (T[:, 0, 0] + T[:, 1, 0]) / 2
        D = 0.5 * (grad_V + grad_V.transpose(0, 2, 1))
        I1 = D[:, 0, 0] + D[:, 1, 1]
        mu = self.mu * (Tm / self.T_0) ** 1.5 * (self.T_0 + self.S) / (Tm + self.S)
        mu_b = self.mu_b * Tm ** 2 / self.T_0 ** 2
        tau = (-mu_b * I1)[:, None, None] * np.eye(d, dtype=self.dt)[None] + (-2 * mu)[:, None, None] * D
        P = self.eos_P(rho, T)
        c = self.eos_c(T)
        # fluxes (fvm_equation.py:210-368)
        Us_f = np.concatenate([mom, rho, Q + P], axis=-1)
        flux = (Us_f * phi_n[:, :, None]).mean(axis=1, dtype=self.dt)
        flux[:, :d] += P.mean(axis=1, dtype=self.dt) * self.normals
        flux[:, :d] += (tau * self.normals[:, :, None]).sum(axis=-2)
        Vm = Vs.mean(axis=1, keepdims=True, dtype=self.dt)
        heat = (tau * Vm * self.normals[:, :, None]).sum(axis=(-1, -2))
        heat = heat - self.kappa * grad_T_n * self.fsize[:, 0]
        flux[:, d + 1] += heat
        vmag = np.sqrt((Vs ** 2).sum(axis=-1))
        vmax = vmag.max(axis=1, keepdims=True)
        cmax = c.max(axis=1)
        M = np.abs(vmax / (cmax + 1e-8))
        vf = np.clip(M, self.v_factor, 1)
        a_vel = vf * cmax + vmax
        a_oth = cmax + vmax
        kt = 0.5 * np.concatenate([a_vel * (mom[:, 0] - mom[:, 1]), a_oth * (rho[:, 0] - rho[:, 1]),
                                   a_oth * (Q[:, 0] - Q[:, 1])], axis=1) * self.fsize
        flux = flux + kt
        # divergence (fvm_equation.py:428-435)
        if return_faces:
            return ell_spmm(*self.Fm, flux), grads, Ufa
        return ell_spmm(*self.Fm, flux), grads


# ---------------------------------------------------------------------------------------------
# State conversion (fvm_equation.py:35-55)
# ---------------------------------------------------------------------------------------------
def state_to_prim(state, dim, C_v):
    mom, rho, Q = state[:, :dim], state[:, dim:dim + 1], state[:, dim + 1:dim + 2]
    V = mom / rho
    T = 1 / C_v * (Q / rho - 0.5 * (V ** 2).sum(axis=1, keepdims=True))
    return np.concatenate([V, rho, T], axis=-1)


def prim_to_state(prim, dim, C_v):
    V, rho, T = prim[:, :dim], prim[:, dim:dim + 1], prim[:, dim + 1:dim + 2]
    return np.concatenate([V * rho, rho, rho * (C_v * T + 0.5 * (V ** 2).sum(axis=-1, keepdims=True))], -1)


# ---------------------------------------------------------------------------------------------
# Integrators (integrators.py)
# ---------------------------------------------------------------------------------------------
TABLEAUS = {
    # integrators.py:216-226
    "RK4": (np.array([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1.0, 0]]),
            np.array([1 / 6, 1 / 3, 1 / 3, 1 / 6]), np.array([0.25] * 4)),
    # integrators.py:228-238
    "RK3_SSP4": (np.array([[0, 0, 0, 0], [0.5, 0, 0, 0], [0.5, 0.5, 0, 0], [1 / 6, 1 / 6, 1 / 6, 0]]),
                 np.array([1 / 6, 1 / 6, 1 / 6, 1 / 2]), np.array([0.25] * 4)),
    # Shu-Osher three-stage SSP-RK3 as a Butcher tableau (restated; the reference only has it in the
    # unreachable integrators_bad.py:13-35)
    "SSP_RK3": (np.array([[0, 0, 0], [1.0, 0, 0], [0.25, 0.25, 0]]),
                np.array([1 / 6, 1 / 6, 2 / 3]), np.array([0.5, 0.5, 0.0])),
}
# The remaining tableaus of integrators.py, as lower-triangular rows (the coefficients are the
# reference's constants and must be the same numbers).
_SSP5_A = [[0.37726891511710], [0.37726891511710, 0.37726891511710],
           [0.16352294089771] * 3, [0.14904059394856, 0.14831273384724, 0.14831273384724, 0.34217696850008]]
_SSP6_A = [[0.28422], [0.28422] * 2, [0.23071] * 3, [0.13416] * 3 + [0.16528],
           [0.13416] * 3 + [0.16528, 0.28422]]
_RK4SSP5_A = [[0.39175222700392], [0.21766909633821, 0.36841059262959],
              [0.08269208670950, 0.13995850206999, 0.25189177424738],
              [0.06796628370320, 0.11503469844438, 0.20703489864929, 0.54497475021237]]
_RK4SSP10_A = [[1 / 6] * k for k in range(1, 5)] + [[1 / 15] * 5 + [1 / 6] * k for k in range(0, 5)]


def _lower(rows):
    s = len(rows) + 1
    A = np.zeros((s, s))
    for i, r in enumerate(rows):
        A[i + 1, :len(r)] = r
    return A


TABLEAUS.update({
    # integrators.py:240-251
    "RK3_SSP5": (_lower(_SSP5_A), np.array([0.19707596384481, 0.11780316509765, 0.11709725193772,
                                            0.27015874934251, 0.29786487010104]), np.full(5, 0.2)),
    # integrators.py:253-265
    "RK3_SSP6": (_lower(_SSP6_A), np.array([0.17016, 0.17016, 0.10198, 0.12563, 0.21604, 0.21604]),
                 np.full(6, 1 / 6)),
    # integrators.py:267-278
    "RK4_SSP5": (_lower(_RK4SSP5_A), np.array([0.14681187618661, 0.24848290924556, 0.10425883036650,
                                               0.27443890091960, 0.22600748319395]), np.full(5, 0.2)),
    # integrators.py:280-296
    "RK4_SSP10": (_lower(_RK4SSP10_A), np.full(10, 0.1),
                  np.array([0.2, 0, 0, 0.3, 0, 0, 0.2, 0, 0.3, 0])),
})


class OracleSolver:
    """Time stepping on the oracle residual; carries ``cell_grads`` exactly as the reference."""

    def __init__(self, residual: OracleResidual, state, dt):
        self.res = residual
        self.state = np.asarray(state, dtype=residual.dt)
        self.grads = None
        self.dt = residual.dt(dt)
        self.hist = []

    def f(self, U):
        prim = state_to_prim(U, self.res.dim, self.res.C_v)
        r, self.grads = self.res.forward(prim, self.grads)
        return r

    def butcher_step(self, name):
        """``Butcher._step`` (integrators.py:369-393)."""
        A, b, _ = TABLEAUS[name]
        dt = self.res.dt
        A, b = A.astype(dt), b.astype(dt)
        U0 = self.state
        k = []
        for i in range(len(b)):
            inc = sum((A[i, j] * k[j] for j in range(i)), np.zeros_like(U0)) if i else 0
            k.append(self.dt * self.f(U0 + inc))
        self.state = U0 + sum(b[i] * k[i] for i in range(len(b)))
        return self.state

    def adapt_step(self, name, atol=2e-3, rtol=2e-3, mtol=1e-6, alphas=(0.8, 0.995), order=4):
        """``ButcherAdapt._step`` + ``Adaptive.update_stepsize`` (integrators.py:42-62, 322-346)."""
        A, b, b2 = TABLEAUS[name]
        dt = self.res.dt
        A, b, b2 = A.astype(dt), b.astype(dt), b2.astype(dt)
        U0 = self.state
        k = []
        for i in range(len(b)):
            inc = sum((A[i, j] * k[j] for j in range(i)), np.zeros_like(U0)) if i else 0
            k.append(self.dt * self.f(U0 + inc))
        hi = sum(b[i] * k[i] for i in range(len(b)))
        lo = sum(b2[i] * k[i] for i in range(len(b)))
        self._update_dt(hi, lo, U0, atol, rtol, mtol, alphas, order)
        self.state = U0 + hi
        return self.state

    def rk3ssp4_step(self):
        """The hand-unrolled ``RK3_SSP4._step`` (integrators.py:72-94)."""
        U0 = self.state
        euler = lambda U: U + self.dt * self.f(U)
        Ua = 0.5 * (U0 + euler(U0))
        Ub = 0.5 * (Ua + euler(Ua))
        Uc = 2 / 3 * U0 + 1 / 6 * (Ub + euler(Ub))
        U1 = 0.5 * (Uc + euler(Uc))
        self._update_dt(U1 - U0, Ub - U0, U0, 2e-3, 2e-3, 1e-6, (0.8, 0.995), 4)
        self.state = U1
        return U1

    def _update_dt(self, hi, lo, U0, atol, rtol, mtol, alphas, order):
        n = lambda x: np.sqrt((x.astype(np.float64) ** 2).sum(axis=0))
        E = (n(hi - lo) / (atol + rtol * n(hi) + mtol * n(U0))).mean()
        fac = 0.9 * E ** (-1 / order)
        alpha = alphas[0] if E > 1 else alphas[1]
        self.dt = self.res.dt(self.dt * (alpha + (1 - alpha) * fac))

    def ab3_step(self):
        """Adams-Bashforth 3 (restated): U += dt/12 (23 f_n - 16 f_{n-1} + 5 f_{n-2})."""
        fn = self.f(self.state)
        self.hist.insert(0, fn)
        self.hist = self.hist[:3]
        if len(self.hist) < 3:
            raise RuntimeError("AB3 needs two start-up steps (use ab3_start)")
        f0, f1, f2 = self.hist
        self.state = self.state + self.dt / 12 * (23 * f0 - 16 * f1 + 5 * f2)
        return self.state

    def ab3_start(self):
        """Two SSP-RK3 start-up steps, recording f(U_n) of each for the AB3 history."""
        for _ in range(2):
            fn = self.f(self.state)
            self.hist.insert(0, fn)
            A, b, _ = TABLEAUS["SSP_RK3"]
            U0 = self.state
            k1 = self.dt * fn
            k2 = self.dt * self.f(U0 + k1)
            k3 = self.dt * self.f(U0 + 0.25 * k1 + 0.25 * k2)
            self.state = U0 + (k1 / 6 + k2 / 6 + 2 * k3 / 3)
        return self.state


def cfl_dt(state, dim, C_v, gamma, inv_h, cfl):
    """dt = cfl * min_i 1 / (inv_h_i (|u_i| + c_i)), FP64 (new; no reference counterpart)."""
    p = state_to_prim(np.asarray(state, np.float64), dim, C_v)
    V, T = p[:, :dim], p[:, dim + 1]
    c = np.sqrt(gamma * C_v * (gamma - 1) * T)
    s = (np.sqrt((V ** 2).sum(axis=1)) + c) * np.asarray(inv_h, np.float64)
    return cfl / s.max()
