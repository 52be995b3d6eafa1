"""The entry seam with the reference's own objects (no GPU).

A user of the reference builds ``ConfigFVM``, ``FVMMesh2D/3D`` and ``Facet`` objects from its own
modules and hands them to ``FVMEquation(cfg, phy_setup, mesh, n_comp, bc_tag, us_init)``
(``time_fvm/fvm_equation.py:377``).  This checks that the B200 host build accepts those objects
unchanged -- the reference mesh object through ``equation._host_mesh``, the reference config and
``Facet`` objects by duck typing -- and produces the same device tables, bit for bit, and the same
physics constants as this package's own objects.  Needs the reference sources
(``FVM_REFERENCE_PATH``); skipped without them.
"""
import os
import sys

import numpy as np
import pytest
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from refimport import import_reference, reference_available  # noqa: E402

pytestmark = pytest.mark.skipif(not reference_available(), reason="needs FVM_REFERENCE_PATH (reference sources)")


def _ref_objects(R, g, dim):
    spec_cells = torch.from_numpy(g["cells"])
    RM, st = R["fvm_mesh"], R["mesh_store"]
    cls = RM.FVMMesh2D if dim == 2 else RM.FVMMesh3D
    mesh = cls(torch.from_numpy(g["vertices"]), spec_cells, torch.from_numpy(g["facets"]),
               torch.from_numpy(g["bc_facet_mask"]), device="cpu")
    cfg = R["config_fvm"].ConfigEllipse()
    cfg.device, cfg.compile, cfg.plot = "cpu", False, False
    if dim == 3:
        cfg.exit_cfg.v_inf = (3.0, 0.0, 0.0)
        cfg.inlet_cfg.v_inf = (3.0, 0.0, 0.0)
    E, Facet = st.FacetBCTypes, st.Facet
    bc = {}
    for i, tg in enumerate(str(t) for t in g["bc_tags"]):
        if tg == "NavierWall":
            bc[i] = Facet([E.Dirich] * dim + [E.Neuman] * 2, [0.0] * dim + [None, None], [None] * dim + [0, 0], tag=tg)
        elif tg in ("Left", "Farfield"):
            bc[i] = Facet([E.Inlet] * (dim + 2), tag=tg)
        else:
            bc[i] = Facet([E.Farfield] * (dim + 2), tag=tg)
    return mesh, cfg, bc


@pytest.mark.parametrize("case", ["c2d", "b3d"])
def test_tables_from_reference_objects(case):
    from conftest import golden_setup
    from fvm_solver_b200 import equation as EQ, tables as tb
    g, spec, T_own, cfg_own = golden_setup(case)
    dim = int(g["dim"])
    R = import_reference()
    mesh, cfg, bc = _ref_objects(R, g, dim)
    T_ref = tb.FVMTables(EQ._host_mesh(mesh), cfg, dim + 2, bc)
    ka, kb = T_ref.kernel, T_own.kernel
    names = [k for k, v in vars(ka).items() if isinstance(v, torch.Tensor)]
    assert len(names) > 10
    for k in names:
        assert torch.equal(getattr(ka, k), getattr(kb, k)), k
    for k in ("G_mats", "flux_mat", "A_face_grad"):
        a, b = getattr(T_ref.ops, k), getattr(T_own.ops, k)
        assert torch.equal(a.coalesce().indices(), b.coalesce().indices()), k
        assert torch.equal(a.coalesce().values(), b.coalesce().values()), k
    # physics constants from the reference's config object and FluidConstitution fields
    phy_ref = (EQ.FluidConstitution2D if dim == 2 else EQ.FluidConstitution3D)(cfg)
    phy_own = (EQ.FluidConstitution2D if dim == 2 else EQ.FluidConstitution3D)(cfg_own)
    pa, pb = phy_ref.physics_struct(cfg), phy_own.physics_struct(cfg_own)
    for f, _ in pa._fields_:
        assert getattr(pa, f) == getattr(pb, f), f


def test_reference_facet_rules_match():
    """The package's ``Facet`` accepts and rejects the same specifications as the reference's."""
    from fvm_solver_b200 import mesh_store as ms
    R = import_reference()
    st = R["mesh_store"]
    for mod in (st, ms):
        E = mod.FacetBCTypes
        ok = [([E.Dirich, E.Neuman], [1.0, None], [None, 0.0]), ([E.Inlet] * 3, None, None),
              ([E.Farfield] * 2, None, None)]
        bad = [([E.Dirich], None, None), ([E.Neuman], [1.0], [0.0]), ([E.Inlet, E.Dirich], [None, 1.0], None),
               ([E.Both], [1.0], [0.0])]
        for et, u, d in ok:
            f = mod.Facet(et, u, d)
            assert np.array_equal(np.isnan(np.asarray(f.U, float)), [v is None for v in (u or [None] * len(et))])
            f.farfield(), f.inlet()
        for et, u, d in bad:
            with pytest.raises(AssertionError):
                f = mod.Facet(et, u, d)
                f.farfield(), f.inlet()
    for et, u, d in ([[st.FacetBCTypes.Dirich, st.FacetBCTypes.Neuman], [1.0, None], [None, 0.0]],):
        a = st.Facet(et, u, d)
        b = ms.Facet([ms.FacetBCTypes[e.name] for e in et], u, d)
        assert a.dirichlet() == b.dirichlet() and a.neumann() == b.neumann()
        assert a.farfield() == b.farfield() and a.inlet() == b.inlet()
