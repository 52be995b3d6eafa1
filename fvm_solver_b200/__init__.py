"""B200-native finite-volume residual and time stepping for compressible Navier-Stokes.

Drop-in for the hot path of Merlotec/fvm_solver: the ELL sparse operators (``sparse.SPMB200``,
``to_sparse``), the residual (``equation.FVMEquation.forward``) and the integrators
(``solvers``), all running on hand-written sm_100a kernels in ``libfvm_b200.so``.
"""
from .config import (BCMode, ChannelCylinderConfig, ConfigBC, ConfigEllipse, ConfigFVM,  # noqa: F401
                      EnsembleCaseConfig, TaylorGreenConfig)
from .mesh_store import Facet, FacetBCTypes  # noqa: F401

__all__ = ["BCMode", "ConfigBC", "ConfigFVM", "ConfigEllipse", "ChannelCylinderConfig", "TaylorGreenConfig",
           "EnsembleCaseConfig", "Facet", "FacetBCTypes"]
