"""Residual seam: ``FluidConstitution2D/3D``, ``FVMCells``, ``FVMEquation``.

Mirrors ``time_fvm/fvm_equation.py`` and ``time_fvm/time_solvers/t_solvers.py:15-42``.

``FVMEquation(cfg, phy_setup, mesh, n_comp, bc_tag, us_init)`` has the reference's signature.
``mesh`` may be this package's ``FVMMesh2D/3D`` or any object with the reference mesh's raw inputs
(``vertices``, ``cells``, ``facets``, ``bc_facet_mask``; e.g. a reference ``FVMMesh2D``): the host
tables are rebuilt from them bit-identically.  ``forward(primatives)`` returns dU/dt through the
fused CUDA residual (``fvm_residual``) and, like the reference, carries the limited cell
gradients (``cell_grads``) into the next call's boundary correction.
"""
from __future__ import annotations

import ctypes as ct

import torch

from . import _lib
from .config import ConfigFVM
from .fvm_mesh import FVMMesh, FVMMesh2D, FVMMesh3D
from types import SimpleNamespace

from .tables import FVMTables, KernelTables, grad_index, row_sizes


class FluidConstitution:
    """Ideal gas with Sutherland viscosity (``fvm_equation.py:16-87``).

    The conversions below are setup/inspection utilities (torch ops); the time loop converts on
    the device inside the stage kernels.
    """
    dim: int

    def __init__(self, cfg: ConfigFVM, dim: int):
        self.device = cfg.device
        self.dim = dim
        self.T_0 = cfg.T_0
        self.mu = cfg.viscosity
        self.mu_b = cfg.visc_bulk
        self.S_const = cfg.S_const
        self.C_v = cfg.C_v
        self.gamma = cfg.gamma
        self.R = self.C_v * (cfg.gamma - 1)

    def state_to_primative(self, state: torch.Tensor):
        d = self.dim
        momentum, rho, Q = state[:, :d], state[:, d:d + 1], state[:, d + 1:d + 2]
        V = momentum / rho
        T = 1 / self.C_v * (Q / rho - 0.5 * V.square().sum(dim=1, keepdim=True))
        return torch.cat([V, rho, T], dim=-1), state

    def primatives_to_state(self, V, rho, T):
        momentum = V * rho
        Q = rho * (self.C_v * T + 0.5 * V.square().sum(dim=-1, keepdim=True))
        return momentum, rho, Q

    def eos_c(self, rho, T):
        return torch.sqrt(self.gamma * self.R * T)

    def eos_P(self, rho, T):
        return self.R * rho * T

    def eos_T(self, rho, P):
        return P / (self.R * rho)

    def physics_struct(self, cfg: ConfigFVM) -> _lib.Physics:
        return _lib.Physics(T_0=self.T_0, mu=self.mu, mu_b=self.mu_b, S_const=self.S_const, C_v=self.C_v,
                            gamma=self.gamma, kappa=cfg.thermal_cond, v_factor=cfg.v_factor,
                            lim_p=cfg.lim_p)


class FluidConstitution2D(FluidConstitution):
    def __init__(self, cfg: ConfigFVM, dim: int = 2):
        super().__init__(cfg, dim)
        assert self.dim == 2, "Only for 2D fluids"


class FluidConstitution3D(FluidConstitution):
    def __init__(self, cfg: ConfigFVM, dim: int = 3):
        super().__init__(cfg, dim)
        assert self.dim == 3, "Only for 3D fluids"


class DeviceMesh:
    """Kernel tables uploaded to one device (record layout), plus the ``fvm_mesh_t`` struct."""

    _struct_fields = [f for f in _lib.MESH_PTR_FIELDS if f not in
                      ("cell_rec", "div_rec", "face_rec", "cell_case", "face_case", "bc_case", "ch_off",
                       "case_mu", "case_mu_b", "case_kappa", "case_active")]

    def __init__(self, kt: KernelTables, device, records: dict | None = None):
        """``records``: precomputed device records (default ``kt.records()``)."""
        self.device = torch.device(device)
        self.dim, self.n_comp, self.n_cells = kt.dim, kt.n_comp, kt.n_cells
        self.n_facets, self.n_bc, self.kg, self.kf = kt.n_facets, kt.n_bc, kt.kg, kt.kf
        self.row, self.grow = row_sizes(kt.dim)
        up = {k: v.contiguous().to(self.device) for k, v in (records or kt.records()).items()}
        for f in self._struct_fields:
            up[f] = getattr(kt, f).contiguous().to(self.device)
        self.t = SimpleNamespace(**up)
        m = _lib.Mesh(dim=kt.dim, n_comp=kt.n_comp, n_cells=kt.n_cells, n_facets=kt.n_facets,
                      n_bc=kt.n_bc, n_char=kt.n_char, kg=kt.kg, kf=kt.kf)
        for f, v in up.items():
            setattr(m, f, _lib.ptr(v))
        self.struct = m

    def work(self) -> "Work":
        return Work(self)

    def bytes(self) -> int:
        return sum(v.numel() * v.element_size() for v in vars(self.t).values())


class Work:
    """Caller-owned scratch of one mesh (``fvm_work_t``)."""

    def __init__(self, dm: DeviceMesh):
        R, dev = dm.row, dm.device
        self.bc_vals = torch.zeros((max(dm.n_bc, 1), R), device=dev)
        self.prims = torch.zeros((dm.n_cells, R), device=dev)
        self.flux = torch.zeros((dm.n_facets, R), device=dev)
        # + 8: the per-part slots of partitioned meshes (fvm_char_partial / char_scale_given)
        self.red = torch.zeros(_lib.FVM_RED_DOUBLES + 8, device=dev, dtype=torch.float64)
        self.struct = _lib.Work(bc_vals=_lib.ptr(self.bc_vals), prims=_lib.ptr(self.prims),
                                flux=_lib.ptr(self.flux), red=_lib.ptr(self.red))


def grads_to_reference(g: torch.Tensor, dim: int) -> torch.Tensor:
    """Limited-gradient rows [N][FVM_GROW] -> the reference's cell_grads layout [N, dim, C]."""
    C = dim + 2
    idx = torch.tensor([[grad_index(dim, d, c) for c in range(C)] for d in range(dim)], device=g.device)
    return g[:, idx]


def _host_mesh(mesh, dim_hint=None) -> FVMMesh:
    if isinstance(mesh, FVMMesh):
        return mesh
    cls = FVMMesh2D if mesh.vertices.shape[1] == 2 else FVMMesh3D
    kw = {}
    if getattr(mesh, "period", None) is not None:
        kw = dict(period=mesh.period, cell_shifts=mesh.cell_shifts, facet_shifts=mesh.facet_shifts)
    return cls(mesh.vertices.float().cpu(), mesh.cells.cpu(), mesh.facets.cpu(), mesh.bc_facet_mask.cpu(), **kw)


class _MeshInfo:
    def __init__(self, n_cells, dim):
        self.n_cells = n_cells
        self.dim = dim


class FVMCells:
    """Conserved state on the device (``t_solvers.py:15-42``)."""

    def __init__(self, n_cells, n_comp, phys_setup: FluidConstitution, init_val=None, device="cuda"):
        self.device = device
        self.phys_setup = phys_setup
        if init_val is None:
            state = torch.zeros(n_cells, n_comp, device=device)
        else:
            assert init_val.shape == (n_cells, n_comp), f"Incorrect us init shape {init_val.shape = }"
            state = init_val.to(device=device, dtype=torch.float32)
        self._state = state.contiguous()
        self.version = 0

    @property
    def state(self) -> torch.Tensor:
        return self._state

    @state.setter
    def state(self, value: torch.Tensor):
        self._state.copy_(value)
        self.version += 1

    def copy_from(self, value: torch.Tensor, non_blocking: bool = False):
        """Set the state from ``value`` (host or device); ``non_blocking`` with a pinned host
        tensor enqueues the copy on the current stream without waiting for it.  (``load`` below
        keeps the reference's meaning: read a saved state file.)"""
        self._state.copy_(value, non_blocking=non_blocking)
        self.version += 1

    def update_cells(self, state_new):
        self.state = state_new

    def get_values(self):
        return self.phys_setup.state_to_primative(self._state)

    def convert_state_to_value(self, state):
        return self.phys_setup.state_to_primative(state)

    def save(self, name="state.pt"):
        torch.save(self._state, name)

    def load(self, name="state.pt"):
        self.state = torch.load(name, weights_only=True).to(self.device)


class FVMEquation:
    """``FVMEquation`` (``fvm_equation.py:371-435``) on the B200 kernels."""

    def __init__(self, cfg: ConfigFVM, phy_setup: FluidConstitution, mesh, n_comp, bc_tag, us_init=None,
                 build_solver: bool = True):
        if getattr(cfg, "backend", "b200") != "b200":
            raise ValueError(f"unknown backend {cfg.backend!r}")
        self.cfg = cfg
        self.phy_setup = phy_setup
        self.device = torch.device(cfg.device)
        if self.device.type != "cuda":
            raise RuntimeError("fvm_solver_b200 runs on CUDA devices only (no CPU fallback)")
        self.lib = _lib.load()
        self.mesh = _host_mesh(mesh)
        if getattr(cfg, "grad_stencil", None):
            self.mesh.widen_gradient_stencil(int(cfg.grad_stencil))
        self.n_comp = n_comp
        assert n_comp == self.mesh.dim + 2, "n_comp must be dim + 2"
        self.tables = FVMTables(self.mesh, cfg, n_comp, bc_tag)
        self.dev = DeviceMesh(self.tables.kernel, self.device)
        self.work = self.dev.work()
        self.phys = phy_setup.physics_struct(cfg)
        N, dim = self.mesh.n_cells, self.mesh.dim
        self.grads = torch.zeros((N, self.dev.grow), device=self.device)
        self.has_grads = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._has_grads_host = False
        self.cells = FVMCells(N, n_comp, init_val=us_init, phys_setup=phy_setup, device=self.device)
        self.t_solver = None
        if build_solver:
            from .solvers import get_solver
            self.t_solver = get_solver(self.cells, self, cfg)

    @classmethod
    def from_kernel_tables(cls, cfg: ConfigFVM, phy_setup: FluidConstitution, kt: KernelTables, us_init,
                           build_solver: bool = True) -> "FVMEquation":
        """Construct from prebuilt kernel tables (e.g. built once and shared with a batch)."""
        self = cls.__new__(cls)
        self.cfg, self.phy_setup = cfg, phy_setup
        self.device = torch.device(cfg.device)
        self.lib = _lib.load()
        self.mesh = _MeshInfo(kt.n_cells, kt.dim)
        self.n_comp = kt.n_comp
        self.tables = None
        self.dev = DeviceMesh(kt, self.device)
        self.work = self.dev.work()
        self.phys = phy_setup.physics_struct(cfg)
        self.grads = torch.zeros((kt.n_cells, self.dev.grow), device=self.device)
        self.has_grads = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._has_grads_host = False
        self.cells = FVMCells(kt.n_cells, kt.n_comp, init_val=us_init, phys_setup=phy_setup, device=self.device)
        self.t_solver = None
        if build_solver:
            from .solvers import get_solver
            self.t_solver = get_solver(self.cells, self, cfg)
        return self

    @property
    def cell_grads(self):
        """Limited cell gradients of the last evaluation [N, dim, C], or None before the first."""
        return grads_to_reference(self.grads, self.mesh.dim) if self._has_grads_host else None

    def reset_gradients(self):
        """Forget the carried gradients (the next evaluation behaves like the reference's first)."""
        self.has_grads.zero_()
        self._has_grads_host = False

    def solve(self):
        self.t_solver.solve()

    def forward(self, primatives: torch.Tensor) -> torch.Tensor:
        """dU/dt [N, C] of the primitives [N, C] (V, rho, T)."""
        prims = primatives.to(device=self.device, dtype=torch.float32).contiguous()
        assert prims.shape == (self.mesh.n_cells, self.n_comp), f"bad primatives shape {tuple(prims.shape)}"
        out = torch.empty_like(prims)
        _lib.check(self.lib.fvm_residual(ct.byref(self.dev.struct), ct.byref(self.phys), _lib.ptr(prims),
                                         _lib.ptr(self.grads), _lib.ptr(self.has_grads), _lib.ptr(out),
                                         ct.byref(self.work.struct), _lib.stream_ptr()), "fvm_residual")
        self._has_grads_host = True
        return out

    def forward_noalloc(self, primatives: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """``forward`` through ``fvm_residual_noalloc``: writes dU/dt into the caller's ``out``.

        For callers that cannot allocate device memory at the call: the library allocates nothing
        (its scratch is a 16 MiB static device array shared by all calls on the device, so calls
        must not overlap on the GPU), and ``primatives`` / ``out`` must already be contiguous
        float32 CUDA tensors of shape [N, C].  Raises ``RuntimeError`` if the mesh needs more
        scratch than the static array holds.
        """
        N, C = self.mesh.n_cells, self.n_comp
        for t in (primatives, out):
            if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and tuple(t.shape) == (N, C)):
                raise ValueError("forward_noalloc needs contiguous float32 CUDA tensors of shape [N, C]")
        _lib.check(self.lib.fvm_residual_noalloc(ct.byref(self.dev.struct), ct.byref(self.phys),
                                                 _lib.ptr(primatives), _lib.ptr(self.grads),
                                                 _lib.ptr(self.has_grads), _lib.ptr(out), _lib.stream_ptr()),
                   "fvm_residual_noalloc")
        self._has_grads_host = True
        return out

    def facet_state(self, primatives: torch.Tensor):
        """The facet attributes the reference's ``FacetCalc.compute_facet`` leaves on ``E_props``
        (``facet_process.py:349-359``) and its consumers read (``Saver.save``,
        ``saving.py:54-57``): ``Vs_facet`` [F, 2, dim], ``rho_facet`` / ``T_facet`` [F, 2, 1],
        ``mom_facet``, ``Q_facet`` and ``phi`` [F, 2] for the primitives ``primatives`` [N, C].

        On demand: one residual evaluation on scratch gradients (first-call semantics, the carried
        gradients are left alone) and one kernel that rebuilds both sides of every facet as the
        facet kernel does.  The hot path stores none of this."""
        from types import SimpleNamespace
        prims = primatives.to(device=self.device, dtype=torch.float32).contiguous()
        dim, C = self.mesh.dim, self.n_comp
        grads = torch.zeros_like(self.grads)
        flag = torch.zeros(1, dtype=torch.int32, device=self.device)
        dudt = torch.empty_like(prims)
        _lib.check(self.lib.fvm_residual(ct.byref(self.dev.struct), ct.byref(self.phys), _lib.ptr(prims),
                                         _lib.ptr(grads), _lib.ptr(flag), _lib.ptr(dudt), ct.byref(self.work.struct),
                                         _lib.stream_ptr()), "fvm_residual")
        U = torch.empty((self.dev.n_facets, 2, C), device=self.device)
        _lib.check(self.lib.fvm_facet_values(ct.byref(self.dev.struct), _lib.ptr(self.work.prims), _lib.ptr(grads),
                                             ct.byref(self.work.struct), _lib.ptr(U), _lib.stream_ptr()),
                   "fvm_facet_values")
        Vs, rho, T = U[:, :, :dim].contiguous(), U[:, :, dim:dim + 1].contiguous(), U[:, :, dim + 1:].contiguous()
        mom, _, Q = self.phy_setup.primatives_to_state(Vs, rho, T)
        phi = None
        if self.tables is not None:
            phi = (Vs * self.tables.normals.to(self.device).unsqueeze(1)).sum(dim=-1)
        return SimpleNamespace(Vs_facet=Vs, rho_facet=rho, T_facet=T, mom_facet=mom, Q_facet=Q, phi=phi,
                               cell_grads=grads_to_reference(grads, dim), dudt=dudt)

    def conservation(self, state: torch.Tensor | None = None) -> torch.Tensor:
        """FP64 totals sum_i vol_i U_i [C] of ``state`` (default: the current cell state)."""
        s = (self.cells.state if state is None else state).contiguous()
        out = torch.empty((1, self.n_comp), dtype=torch.float64, device=self.device)
        _lib.check(self.lib.fvm_conservation(ct.byref(self.dev.struct), _lib.ptr(s), _lib.ptr(out),
                                             ct.byref(self.work.struct), _lib.stream_ptr()), "fvm_conservation")
        return out[0]
