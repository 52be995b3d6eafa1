"""Solver configuration, mirroring the reference's ``ConfigFVM`` dataclass.

Reference: ``time_fvm/config_fvm.py:6-67`` (``BCMode``, ``ConfigBC``, ``ConfigFVM``) and the
presets at ``time_fvm/config_fvm.py:71-178``.  Every field of the reference keeps its name and
meaning so an existing config object can be handed to this package unchanged.  Added fields:

* ``backend`` -- ``"b200"`` (the only backend; kept so callers can select it explicitly).
* ``grad_stencil`` -- least-squares gradient stencil slots per cell, the cell included (at most
  16): None keeps the reference's face-neighbour stencil (dim + 2 slots); a larger value adds the
  nearest second-ring cells (``fvm_mesh.FVMMesh.widen_gradient_stencil``).
* ``cfl`` -- when set, the time step is ``cfl * min_i h_i / (|u_i| + c_i)`` recomputed on the
  device every step (FP64 min-reduction); ``h_i = vol_i / max face area``.  The reference has no
  CFL control (fixed ``dt`` or error-adaptive ``dt``); this is a new, documented extension.

The three workload presets below (``ChannelCylinderConfig``, ``TaylorGreenConfig``,
``EnsembleCaseConfig``) state the physical mapping (Mach, Reynolds, Prandtl -> ``viscosity``,
``thermal_cond``) that both the CUDA path and the oracle use.
"""
from __future__ import annotations

import math
from abc import ABC
from dataclasses import dataclass, field
from enum import Enum


class BCMode(Enum):
    """Boundary-condition family of a characteristic-type boundary (``config_fvm.py:6-9``)."""
    Isentropic = "Isentropic"
    Characteristic = "characteristic"
    Farfield = "Farfield"


class ConfigBC(ABC):
    """Far-field state of an inlet / exit boundary (``config_fvm.py:12-19``).

    ``v_n_inf`` is inward-positive in 2D; 3D configs give ``v_inf`` as a vector.
    """
    mode: BCMode
    v_n_inf: float
    v_t_inf: float
    v_inf: tuple
    rho_inf: float
    T_inf: float


@dataclass
class ConfigFVM(ABC):
    device: str = "cuda"
    compile: bool = False
    profile: bool = False

    problem_setup: str | None = None
    N_comp: int = 4

    # Temporal solver parameters
    solver_name: str = "Butcher_adapt"
    solver_extra: str = "RK3_SSP4"
    dt: float | None = None
    n_iter: int | None = None

    # mesh parameters
    min_A: float | None = None
    max_A: float | None = None
    lnscale: float | None = None

    # Save configuration
    plot: bool = False
    plot_t: float | None = None
    save_t: float | None = None
    save_dir: str | None = None
    exact_interval: bool = False
    print_i: int | None = None
    end_t: float | None = None

    # Physical parameters
    T_0: float | None = None
    viscosity: float | None = None
    visc_bulk: float | None = None
    thermal_cond: float | None = None
    S_const: float | None = None
    gamma: float | None = None
    C_v: float | None = None

    # Stability parameters
    v_factor: float = 0.1
    lim_p: int = 4
    lim_K: float = 0.1

    # Boundary configuration
    exit_cfg: ConfigBC | None = None
    inlet_cfg: ConfigBC | None = None

    # Additions of this package
    backend: str = "b200"
    cfl: float | None = None
    grad_stencil: int | None = None

    @property
    def R(self) -> float:
        return self.C_v * (self.gamma - 1)


@dataclass
class CharacteristicBC(ConfigBC):
    """A characteristic far-field boundary (the reference's ``EllipseFarfield``/``EllipseInlet``)."""
    mode: BCMode = BCMode.Characteristic
    v_n_inf: float = 0.0
    v_t_inf: float = 0.0
    v_inf: tuple = (0.0, 0.0, 0.0)
    rho_inf: float = 1.0
    T_inf: float = 100.0


# ---------------------------------------------------------------------------------------------
# Reference presets (``config_fvm.py:94-123``), kept for parity tests.
# ---------------------------------------------------------------------------------------------
@dataclass
class ConfigEllipse(ConfigFVM):
    problem_setup: str | None = "ellipse"
    dt: float | None = 1e-4
    n_iter: int | None = 50000
    min_A: float | None = 0.25e-3
    max_A: float | None = 0.5e-3
    lnscale: float | None = 2
    plot_t: float | None = 0.5
    save_t: float | None = 0.5
    print_i: int | None = 500
    end_t: float | None = 20
    T_0: float | None = 100
    viscosity: float | None = 1e-3
    visc_bulk: float | None = 10e-3
    thermal_cond: float | None = 1e-6
    S_const: float | None = 110.4
    gamma: float | None = 1.2
    C_v: float | None = 2

    def __post_init__(self):
        self.exit_cfg = CharacteristicBC(v_n_inf=-5.5, v_t_inf=0.0, rho_inf=1.0, T_inf=100.0)
        self.inlet_cfg = CharacteristicBC(v_n_inf=5.5, v_t_inf=0.0, rho_inf=1.0, T_inf=100.0)


# ---------------------------------------------------------------------------------------------
# Workload presets.
# ---------------------------------------------------------------------------------------------
def _gas(gamma: float, C_v: float, T: float) -> float:
    """Speed of sound of the ideal gas, c = sqrt(gamma * R * T), R = C_v (gamma - 1)."""
    return math.sqrt(gamma * C_v * (gamma - 1.0) * T)


@dataclass
class ChannelCylinderConfig(ConfigFVM):
    """2D channel [0,2]x[0,1] with a cylinder; freestream Mach / Reynolds on the diameter.

    mu_0 = rho U D / Re at T_0 = T_inf; kappa = gamma C_v mu_0 / Pr (constant, as in the reference's
    ``Heating`` term); bulk viscosity = mu_0; Sutherland constant 110.4 (the reference's value).
    Left = inlet, right = exit (both characteristic), walls and cylinder = no-slip.
    """
    problem_setup: str | None = "channel_cylinder"
    N_comp: int = 4
    solver_name: str = "Butcher"
    solver_extra: str = "SSP_RK3"
    cfl: float | None = 0.5
    dt: float | None = 1e-4
    n_iter: int | None = 500
    mach: float = 0.3
    reynolds: float = 200.0
    prandtl: float = 0.72
    radius: float = 0.1
    center: tuple = (0.5, 0.5)
    rho_inf: float = 1.0
    T_inf: float = 100.0
    T_0: float | None = 100.0
    S_const: float | None = 110.4
    gamma: float | None = 1.4
    C_v: float | None = 2.0
    noise: float = 1e-3

    def __post_init__(self):
        self.T_0 = self.T_inf
        U = self.mach * _gas(self.gamma, self.C_v, self.T_inf)
        self.u_inf = U
        mu0 = self.rho_inf * U * (2.0 * self.radius) / self.reynolds
        self.viscosity = mu0
        self.visc_bulk = mu0
        self.thermal_cond = self.gamma * self.C_v * mu0 / self.prandtl
        self.inlet_cfg = CharacteristicBC(v_n_inf=U, v_t_inf=0.0, rho_inf=self.rho_inf, T_inf=self.T_inf)
        self.exit_cfg = CharacteristicBC(v_n_inf=-U, v_t_inf=0.0, rho_inf=self.rho_inf, T_inf=self.T_inf)


@dataclass
class SphereConfig(ConfigFVM):
    """3D flow over a sphere of radius 0.5 in [-5, 15] x [-5, 5]^2; freestream along +x, Mach /
    Reynolds on the diameter.  Gas and transport as ``ChannelCylinderConfig``; the box faces are
    characteristic boundaries with the freestream velocity vector, the sphere is a no-slip wall.
    """
    problem_setup: str | None = "sphere"
    N_comp: int = 5
    solver_name: str = "Butcher"
    solver_extra: str = "SSP_RK3"
    cfl: float | None = 0.5
    dt: float | None = 1e-4
    n_iter: int | None = 500
    mach: float = 0.3
    reynolds: float = 200.0
    prandtl: float = 0.72
    radius: float = 0.5
    rho_inf: float = 1.0
    T_inf: float = 100.0
    T_0: float | None = 100.0
    S_const: float | None = 110.4
    gamma: float | None = 1.4
    C_v: float | None = 2.0
    noise: float = 1e-3

    def __post_init__(self):
        self.T_0 = self.T_inf
        U = self.mach * _gas(self.gamma, self.C_v, self.T_inf)
        self.u_inf = U
        mu0 = self.rho_inf * U * (2.0 * self.radius) / self.reynolds
        self.viscosity = mu0
        self.visc_bulk = mu0
        self.thermal_cond = self.gamma * self.C_v * mu0 / self.prandtl
        v = (U, 0.0, 0.0)
        self.inlet_cfg = CharacteristicBC(v_inf=v, rho_inf=self.rho_inf, T_inf=self.T_inf)
        self.exit_cfg = CharacteristicBC(v_inf=v, rho_inf=self.rho_inf, T_inf=self.T_inf)


@dataclass
class TaylorGreenConfig(ConfigFVM):
    """3D periodic box [0, 2 pi L]^3, Taylor-Green vortex at Mach / Reynolds on V0 and L = 1."""
    problem_setup: str | None = "taylor_green"
    N_comp: int = 5
    solver_name: str = "Butcher"
    solver_extra: str = "RK4"
    cfl: float | None = 0.5
    dt: float | None = 1e-4
    n_iter: int | None = 200
    mach: float = 0.1
    reynolds: float = 1600.0
    prandtl: float = 0.71
    rho_0: float = 1.0
    T_inf: float = 100.0
    T_0: float | None = 100.0
    S_const: float | None = 110.4
    gamma: float | None = 1.4
    C_v: float | None = 2.0

    def __post_init__(self):
        self.T_0 = self.T_inf
        V0 = self.mach * _gas(self.gamma, self.C_v, self.T_inf)
        self.v0 = V0
        mu0 = self.rho_0 * V0 * 1.0 / self.reynolds
        self.viscosity = mu0
        self.visc_bulk = mu0
        self.thermal_cond = self.gamma * self.C_v * mu0 / self.prandtl


@dataclass
class EnsembleCaseConfig(ChannelCylinderConfig):
    """One member of the batched 2D ensemble (channel-cylinder family, per-case parameters)."""
    problem_setup: str | None = "ensemble_case"
    solver_name: str = "AB3"
    solver_extra: str = "SSP_RK3"
    n_iter: int | None = 2000
    n_cells_target: int = 10000
