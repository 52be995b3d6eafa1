"""Boundary-facet specification, mirroring ``time_fvm/mesh_utils/mesh_store.py:5-59``.

A ``Facet`` lists, per state component, which boundary treatment applies (Dirichlet value,
Neumann normal gradient, or membership of a characteristic inlet / exit boundary).  The same
consistency rules as the reference are enforced with the same ``AssertionError`` behaviour.
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import Flag, auto


class FacetBCTypes(Flag):
    Dirich = auto()
    Neuman = auto()
    Both = Dirich | Neuman
    Farfield = auto()
    Inlet = auto()


@dataclass
class Facet:
    edge_type: list
    U: list | None = None
    dUdn: list | None = None
    euler_wall: bool = False
    tag: str | None = None

    def __post_init__(self):
        if self.U is None:
            self.U = [None] * len(self.edge_type)
        if self.dUdn is None:
            self.dUdn = [None] * len(self.edge_type)

        for e, u, dudn in zip(self.edge_type, self.U, self.dUdn, strict=True):
            if FacetBCTypes.Dirich in e:
                assert u is not None, "Dirichlet BC requires a value."
                assert dudn is None, "Dirichlet BC does not require a gradient."
            if FacetBCTypes.Neuman in e:
                assert dudn is not None, "Neumann BC requires a gradient."
                assert u is None, "Neumann BC does not require a value."

        self.U = [float("nan") if u is None else u for u in self.U]
        self.dUdn = [float("nan") if d is None else d for d in self.dUdn]

    def dirichlet(self):
        return [FacetBCTypes.Dirich in e for e in self.edge_type]

    def neumann(self):
        return [FacetBCTypes.Neuman in e for e in self.edge_type]

    def farfield(self) -> bool:
        farfield = [FacetBCTypes.Farfield in e for e in self.edge_type]
        is_farfield = all(farfield)
        assert is_farfield or not any(farfield), f"All boundary must be farfield if any are: {farfield}"
        return is_farfield

    def inlet(self) -> bool:
        inlet = [FacetBCTypes.Inlet in e for e in self.edge_type]
        is_inlet = all(inlet)
        assert is_inlet or not any(inlet), f"All boundary must be inlet if any are: {inlet}"
        return is_inlet


def wall_facet(dim: int, tag: str = "NavierWall") -> Facet:
    """No-slip wall: Dirichlet V = 0, Neumann d(rho)/dn = dT/dn = 0 (``run_fvm.py:89-90``)."""
    E = FacetBCTypes
    return Facet([E.Dirich] * dim + [E.Neuman, E.Neuman], [0.0] * dim + [None, None],
                 [None] * dim + [0.0, 0.0], tag=tag)


def inlet_facet(dim: int, tag: str = "Left") -> Facet:
    return Facet([FacetBCTypes.Inlet] * (dim + 2), tag=tag)


def farfield_facet(dim: int, tag: str = "Right") -> Facet:
    return Facet([FacetBCTypes.Farfield] * (dim + 2), tag=tag)


def default_bc_tags(edge_tags, dim: int) -> dict:
    """Map mesh boundary tags to BC specs the way ``run_fvm.init_conds_ellipses`` does."""
    bc = {}
    for i, tg in enumerate(edge_tags):
        if tg == "NavierWall":
            bc[i] = wall_facet(dim, tg)
        elif tg in ("Left", "Farfield"):
            bc[i] = inlet_facet(dim, tg)
        elif tg == "Right":
            bc[i] = farfield_facet(dim, tg)
        else:
            raise ValueError(f"Unknown edge tag {tg}")
    return bc
