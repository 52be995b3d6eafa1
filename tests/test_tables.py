"""Host table build: bit-exact against the reference's packed ELL operators (golden vectors)."""
import numpy as np
import torch

from fvm_solver_b200 import tables as tb


def test_ell_operators_bit_exact(golden):
    g, spec, T, cfg = golden
    for name, A in [("G", T.ops.G_mats), ("flux", T.ops.flux_mat), ("Afg", T.ops.A_face_grad),
                    ("Abc", T.ops.A_bc), ("Acorr", T.ops.A_corr)]:
        v, c = tb.coo_to_ell(A)
        assert np.array_equal(v.numpy(), g[f"ell_{name}_vals"]), name
        assert np.array_equal(c.numpy(), g[f"ell_{name}_cols"]), name
    assert np.array_equal(T.ops.b_face_grad.numpy(), g["b_face_grad"])
    # b_bc is uninitialised (torch.empty) on characteristic rows in the reference: compare the rest
    m = (T.bc.dirich_mask | T.bc.neumann_mask).reshape(-1).numpy()
    assert np.array_equal(T.ops.b_bc.numpy()[m], g["b_bc"][m])


def test_kernel_tables_consistent(golden):
    """The slot-major kernel tables encode the same operators as the reference-format ones."""
    g, spec, T, cfg = golden
    K = T.kernel
    N, dim = K.n_cells, K.dim
    gv = g["ell_G_vals"].reshape(N, dim, -1)
    gc = g["ell_G_cols"].reshape(N, dim, -1)
    assert np.array_equal(K.g_vals.numpy(), gv.transpose(1, 2, 0))
    assert np.array_equal(K.g_cols.numpy(), gc[:, 0].T)
    assert np.array_equal(K.f_vals.numpy(), g["ell_flux_vals"].T)
    assert np.array_equal(K.f_cols.numpy(), g["ell_flux_cols"].T)
    # neighbour slots decode to neigh_combine
    slots = np.stack([(K.nb_slot.numpy() >> (4 * j)) & 15 for j in range(dim + 1)], 1)
    assert np.all((K.nb_slot.numpy() >> 24) == K.kg)
    nb = np.take_along_axis(K.g_cols.numpy().T, slots, 1)
    assert np.array_equal(nb, T.neigh_combine.numpy())


def test_coo_to_ell_overflow():
    A = torch.sparse_coo_tensor(torch.tensor([[0, 0, 1], [0, 1, 1]]), torch.ones(3), (2, 2))
    try:
        tb.coo_to_ell(A, K=1)
    except ValueError:
        return
    raise AssertionError("expected ValueError")


def test_device_records_encode_tables(golden):
    """The packed device records hold the same operators as the semantic kernel tables."""
    g, spec, T, cfg = golden
    K = T.kernel
    R = K.records()
    dim, N, F, kg = K.dim, K.n_cells, K.n_facets, K.kg
    cell, face, div = R["cell_rec"], R["face_rec"], R["div_rec"]
    # compact record: the kg - 1 neighbour columns (padded to 4), the cell's own slot in bits
    # 28..30 of the first, then the weights
    assert torch.equal(cell[:, 4:4 + dim * kg].reshape(N, dim, kg), K.g_vals.permute(2, 0, 1))
    nb = cell[:, :kg - 1].contiguous().view(torch.int32).long()
    own = (nb[:, 0] >> 28) & 7
    nb[:, 0] &= (1 << 28) - 1
    cols = torch.empty((N, kg), dtype=torch.long)
    for k in range(kg):
        cols[:, k] = torch.where(k < own, nb[:, min(k, kg - 2)],
                                 torch.where(k == own, torch.arange(N), nb[:, max(k - 1, 0)]))
    assert torch.equal(cols, K.g_cols.t().long())
    o = 4 + dim * kg
    assert torch.equal(cell[:, o:o + (dim + 1) * dim].reshape(N, dim + 1, dim), K.disp.permute(2, 0, 1))
    assert torch.equal(cell[:, o + (dim + 1) * dim], K.eps)
    assert torch.equal(div[:, :K.kf], K.f_vals.t())
    assert torch.equal(div[:, dim + 1:dim + 1 + K.kf].contiguous().view(torch.int32), K.f_cols.t())
    codes = face[:, :2].contiguous().view(torch.int32)
    bc = K.bc_face.long()
    # interior facets: both cells; boundary facets: the cell on one side, -1 - b on the other
    interior = torch.ones(F, dtype=torch.bool)
    interior[bc] = False
    assert torch.equal(codes[interior], K.fcell[interior])
    side = K.bc_side.long()
    assert torch.equal(codes[bc, side], -1 - torch.arange(K.n_bc, dtype=torch.int32))
    assert torch.equal(codes[bc, 1 - side], K.bc_cell)
    assert torch.equal(face[:, 2].abs(), K.inv_d.abs()) and torch.equal(face[:, 3], K.fsize)
    inner = K.fbc < 0
    first = K.fcell[:, 0] < K.fcell[:, 1]
    assert torch.equal(face[inner, 2] > 0, first[inner])      # sign: order of the row's two terms
    # side displacements reproduce cent_to_facet_disp through cell_to_facet
    for j in range(dim + 1):
        f = K.c2f[j].long()
        s_ = ((K.side >> j) & 1).long()
        off = 4 + 2 * dim + s_[:, None] * dim + torch.arange(dim)[None, :]
        assert torch.equal(face[f[:, None], off], K.disp[j].t())


def test_sphere_box_mesh():
    """The 3D sphere-in-box generator: requested size, tags, cells outside the sphere, valid tables."""
    import collections
    import numpy as np
    from fvm_solver_b200 import meshgen as mg, workloads as W
    spec = mg.sphere_box(20000, seed=3)
    assert 0.6 * 20000 < spec.n_cells < 1.6 * 20000
    tags = collections.Counter(spec.bc_tags)
    assert set(tags) == {"NavierWall", "Left", "Right", "Farfield"}
    P = spec.vertices.double().numpy()[spec.cells.long().numpy()]
    assert np.all(np.linalg.norm(P.mean(axis=1), axis=1) > 0.5)
    case = W.sphere(20000, seed=3, device="cpu")
    kt = case.tables().kernel
    assert kt.dim == 3 and kt.n_char > 0 and kt.n_bc == len(spec.bc_tags)
    assert bool((kt.volumes > 0).all())


def test_device_mesh_struct_on_host():
    """The fvm_mesh_t struct fills every pointer field from the tables (built on the CPU here)."""
    from conftest import golden_setup
    from fvm_solver_b200.equation import DeviceMesh
    g, spec, tables, cfg = golden_setup("c2d")
    dm = DeviceMesh(tables.kernel, "cpu")
    m = dm.struct
    for f in ("cell_rec", "div_rec", "face_rec", "inv_h", "volumes", "bc_cell", "bc_kind", "ch_cell"):
        assert getattr(m, f), f
    assert m.n_cases == 0 and not m.case_active and m.n_owned == 0 and m.char_scale_given == 0
    assert m.n_cells == tables.kernel.n_cells and m.kg == tables.kernel.kg


def test_widened_gradient_stencil_exact_for_linear_fields():
    """Widened least-squares stencils (config 2's 'gradient stencil width up to 16'; the reference's
    is dim + 2): every width reproduces the gradient of a linear field exactly (to FP32 rounding,
    1e-4 absolute on unit-size coefficients) and a constant field's gradient is zero on a periodic
    box; rows hold at most the requested slots, the face neighbours and the cell itself always."""
    import numpy as np
    import torch
    from fvm_solver_b200 import fvm_mesh as fm, meshgen as mg
    for spec in (mg.box3d(6, seed=4), mg.channel_cylinder(h=0.05, seed=3), mg.periodic_box(7, seed=5)):
        dim = spec.dim
        for width in (None, 9, 16):
            m = fm.mesh_from_spec(spec, grad_stencil=width)
            N = m.n_cells
            G = [m.gradient_coo(d).coalesce() for d in range(dim)]
            nnz = torch.bincount(G[0].indices()[0], minlength=N)
            assert int(nnz.min()) >= dim + 2 and int(nnz.max()) <= (width or dim + 2)
            a = np.array([0.7, -1.3, 0.4][:dim])
            if spec.period is None:
                f = np.concatenate([m.centroids.double().numpy() @ a,
                                    m.midpoints[m.bc_facet_mask].double().numpy() @ a])
                want = a
            else:
                f, want = np.ones(N), np.zeros(dim)
            for d in range(dim):
                y = torch.sparse.mm(G[d].double(), torch.from_numpy(f)[:, None]).numpy()[:, 0]
                assert np.abs(y - want[d]).max() < 1e-4
