"""Boundary-facet specification: the ``Facet`` / ``FacetBCTypes`` interface of the reference
(``time_fvm/mesh_utils/mesh_store.py:5-59``), which callers build and pass as ``bc_tags``.

The table build (``tables.bc_spec_from_tags``) only reads ``dirichlet()``, ``neumann()``, ``U``,
``dUdn``, ``farfield()`` and ``inlet()``, so the reference's own ``Facet`` objects can be passed in
unchanged (duck typing).  This module's ``Facet`` carries the same fields for callers without the
reference installed.  Its rules, per state component c of a boundary group:

* a Dirichlet component needs a value ``U[c]`` and takes no normal gradient;
* a Neumann component needs a normal gradient ``dUdn[c]`` and takes no value;
* characteristic inlet / exit membership (``Inlet`` / ``Farfield``) holds for every component of
  the group or for none.

A broken rule raises ``AssertionError`` (the reference's behaviour); lists of different lengths
raise ``ValueError``.  Unset values and gradients are stored as NaN.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from enum import Flag, auto


class FacetBCTypes(Flag):
    Dirich = auto()
    Neuman = auto()
    Both = Dirich | Neuman
    Farfield = auto()
    Inlet = auto()


def _check_component(c: int, kind: FacetBCTypes, value, grad) -> None:
    """The value / gradient a component's treatment requires (and forbids)."""
    if kind & FacetBCTypes.Dirich:
        if value is None or grad is not None:
            raise AssertionError(f"component {c}: a Dirichlet boundary takes a value and no gradient "
                                 f"(got value={value!r}, gradient={grad!r})")
    if kind & FacetBCTypes.Neuman:
        if grad is None or value is not None:
            raise AssertionError(f"component {c}: a Neumann boundary takes a gradient and no value "
                                 f"(got value={value!r}, gradient={grad!r})")


def _all_or_none(kinds, flag: FacetBCTypes, what: str) -> bool:
    hits = sum(1 for k in kinds if k & flag)
    if 0 < hits < len(kinds):
        raise AssertionError(f"{what}: {hits} of {len(kinds)} components are {what}; it must be all or none")
    return hits == len(kinds)


@dataclass
class Facet:
    edge_type: list
    U: list | None = None
    dUdn: list | None = None
    euler_wall: bool = False
    tag: str | None = None

    def __post_init__(self):
        n = len(self.edge_type)
        values = [None] * n if self.U is None else list(self.U)
        grads = [None] * n if self.dUdn is None else list(self.dUdn)
        if len(values) != n or len(grads) != n:
            raise ValueError(f"edge_type has {n} components, U {len(values)}, dUdn {len(grads)}")
        for c in range(n):
            _check_component(c, self.edge_type[c], values[c], grads[c])
        self.U = [math.nan if v is None else v for v in values]
        self.dUdn = [math.nan if g is None else g for g in grads]

    def dirichlet(self) -> list:
        return [bool(k & FacetBCTypes.Dirich) for k in self.edge_type]

    def neumann(self) -> list:
        return [bool(k & FacetBCTypes.Neuman) for k in self.edge_type]

    def farfield(self) -> bool:
        return _all_or_none(self.edge_type, FacetBCTypes.Farfield, "farfield")

    def inlet(self) -> bool:
        return _all_or_none(self.edge_type, FacetBCTypes.Inlet, "inlet")


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
