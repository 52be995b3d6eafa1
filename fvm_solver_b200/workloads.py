"""Workload definitions: meshes, boundary tags and initial conditions of the benchmarked cases.

* ``taylor_green``     -- 3D periodic box [0, 2 pi]^3 (jittered-grid Delaunay, jitter 0.2 h),
                          Taylor-Green vortex at Mach 0.1 / Re 1600, RK4 at CFL 0.5.
* ``channel_cylinder`` -- 2D channel [0,2]x[0,1] with a cylinder r = 0.1 at (0.5, 0.5), edge
                          0.02 (~11k triangles), Mach 0.3 / Re 200 on the diameter, uniform
                          freestream + seeded Gaussian density noise 1e-3, SSP-RK3 at CFL 0.5.
* ``ensemble_case``    -- one member of the batched 2D ensemble (per-case seeded geometry and
                          flow parameters; AB3 after an SSP-RK3 start).

Initial conditions are built in FP64 on the host and rounded once to FP32.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import config as cf
from . import meshgen as mg
from .mesh_store import default_bc_tags


def conserved(prim: np.ndarray, dim: int, C_v: float) -> np.ndarray:
    V, rho, T = prim[:, :dim], prim[:, dim:dim + 1], prim[:, dim + 1:dim + 2]
    return np.concatenate([V * rho, rho, rho * (C_v * T + 0.5 * (V ** 2).sum(1, keepdims=True))], 1)


def cell_centroids(spec: mg.MeshSpec) -> np.ndarray:
    pts = spec.vertices.numpy().astype(np.float64)[spec.cells.numpy()]
    if spec.cell_shifts is not None:
        pts = pts + spec.cell_shifts.numpy() * spec.period
    return pts.mean(1)


@dataclass
class Case:
    spec: mg.MeshSpec
    cfg: cf.ConfigFVM
    bc_tags: dict
    state0: torch.Tensor          # [N, C] float32 conserved
    name: str

    @property
    def dim(self) -> int:
        return self.spec.dim

    def equation(self):
        from .equation import FVMEquation, FluidConstitution2D, FluidConstitution3D
        phy = FluidConstitution2D(self.cfg) if self.dim == 2 else FluidConstitution3D(self.cfg)
        return FVMEquation(self.cfg, phy, self.spec, self.dim + 2, self.bc_tags, us_init=self.state0)

    def tables(self):
        from .fvm_mesh import mesh_from_spec
        from .tables import FVMTables
        return FVMTables(mesh_from_spec(self.spec, grad_stencil=getattr(self.cfg, "grad_stencil", None)),
                         self.cfg, self.dim + 2, self.bc_tags)


def taylor_green(n: int = 66, seed: int = 0, device: str = "cuda", **cfg_kw) -> Case:
    """Periodic box with n^3 jittered points (n = 66 -> ~1.96 M tetrahedra)."""
    spec = mg.periodic_box(n=n, seed=seed)
    cfg = cf.TaylorGreenConfig(device=device, **cfg_kw)
    x = cell_centroids(spec)
    V0, rho0, T0 = cfg.v0, cfg.rho_0, cfg.T_inf
    R = cfg.C_v * (cfg.gamma - 1)
    p0 = rho0 * R * T0
    X, Y, Z = x[:, 0], x[:, 1], x[:, 2]
    u = V0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -V0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    p = p0 + rho0 * V0 ** 2 / 16.0 * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    T = np.full_like(u, T0)
    rho = p / (R * T)
    prim = np.stack([u, v, w, rho, T], 1)
    st = torch.from_numpy(conserved(prim, 3, cfg.C_v).astype(np.float32))
    return Case(spec, cfg, {}, st, f"taylor_green_n{n}")


def channel_cylinder(h: float = 0.02, seed: int = 0, device: str = "cuda", radius: float = 0.1,
                     center=(0.5, 0.5), mach: float = 0.3, reynolds: float = 200.0, n_cells: int | None = None,
                     **cfg_kw) -> Case:
    if n_cells is not None:
        spec = mg.channel_cylinder_cells(n_cells, radius=radius, center=center, seed=seed)
    else:
        spec = mg.channel_cylinder(h=h, radius=radius, center=center, seed=seed)
    cfg = cf.ChannelCylinderConfig(device=device, radius=radius, center=tuple(center), mach=mach,
                                   reynolds=reynolds, **cfg_kw)
    N = spec.n_cells
    g = torch.Generator().manual_seed(seed)
    noise = torch.randn(N, generator=g, dtype=torch.float64).numpy()
    prim = np.zeros((N, 4))
    prim[:, 0] = cfg.u_inf
    prim[:, 2] = cfg.rho_inf * (1.0 + cfg.noise * noise)
    prim[:, 3] = cfg.T_inf
    st = torch.from_numpy(conserved(prim, 2, cfg.C_v).astype(np.float32))
    return Case(spec, cfg, default_bc_tags(spec.bc_tags, 2), st, f"channel_cylinder_{N}")


def ensemble_params(case_index: int, base_seed: int = 1234) -> dict:
    """Per-case parameters of the batched ensemble (seeded): cells log-uniform in [2k, 60k]."""
    rng = np.random.default_rng(base_seed + case_index)
    return dict(n_cells=int(round(math.exp(rng.uniform(math.log(2000), math.log(60000))))),
                radius=float(rng.uniform(0.05, 0.15)),
                center=(float(rng.uniform(0.3, 0.8)), float(rng.uniform(0.35, 0.65))),
                mach=float(rng.uniform(0.2, 0.6)), reynolds=float(rng.uniform(100, 1000)),
                seed=int(base_seed + case_index))


def ensemble_case(case_index: int, device: str = "cuda", base_seed: int = 1234, **cfg_kw) -> Case:
    p = ensemble_params(case_index, base_seed)
    c = channel_cylinder(device=device, solver_name="AB3", solver_extra="SSP_RK3", **p, **cfg_kw)
    c.name = f"ensemble_{case_index}"
    return c


def sphere(n_cells: int = 500_000, seed: int = 0, device: str = "cuda", mach: float = 0.3, reynolds: float = 200.0,
           **cfg_kw) -> Case:
    """3D flow over a sphere (radius 0.5, box [-5, 15] x [-5, 5]^2): uniform freestream along +x with
    seeded Gaussian density noise of amplitude 1e-3."""
    spec = mg.sphere_box(n_cells, seed=seed)
    cfg = cf.SphereConfig(device=device, mach=mach, reynolds=reynolds, **cfg_kw)
    N = spec.n_cells
    g = torch.Generator().manual_seed(seed)
    noise = torch.randn(N, generator=g, dtype=torch.float64).numpy()
    prim = np.zeros((N, 5))
    prim[:, 0] = cfg.u_inf
    prim[:, 3] = cfg.rho_inf * (1.0 + cfg.noise * noise)
    prim[:, 4] = cfg.T_inf
    st = torch.from_numpy(conserved(prim, 3, cfg.C_v).astype(np.float32))
    return Case(spec, cfg, default_bc_tags(spec.bc_tags, 3), st, f"sphere_{N}")


def sphere_params(case_index: int, base_seed: int = 5678, cells=(300_000, 800_000)) -> dict:
    """Per-case parameters of the 3D sphere family (seeded): cells uniform in ``cells``, Mach
    0.2-0.4, Reynolds 100-400."""
    rng = np.random.default_rng(base_seed + case_index)
    return dict(n_cells=int(rng.uniform(*cells)), mach=float(rng.uniform(0.2, 0.4)),
                reynolds=float(rng.uniform(100, 400)), seed=int(base_seed + case_index))


def sphere_case(case_index: int, device: str = "cuda", base_seed: int = 5678, cells=(300_000, 800_000),
                **cfg_kw) -> Case:
    c = sphere(device=device, **sphere_params(case_index, base_seed, cells), **cfg_kw)
    c.name = f"sphere_{case_index}"
    return c
