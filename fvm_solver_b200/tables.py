"""Operator and boundary tables assembled on the host, in two forms.

1. **Reference-format operators** (``ReferenceOperators``): the sparse matrices the reference
   assembles in ``MeshCache`` / ``BoundarySetter`` -- ``G_mats`` (``facet_process.py:76-79``),
   ``flux_mat`` (``:200-226``), ``A_face_grad``/``b_face_grad`` (``:114-198``), ``A_bc``/``b_bc``
   (``facet_boundary.py:238-280``) and ``A_corr`` (``:170-236``) -- with the same torch CPU
   operations, so their ELL packing (``csr_to_ell``, ``ell_kernel.py:225-256``) is bit-identical.
   They back the ``SPM`` drop-in and the bit-exactness tests.

2. **Kernel tables** (``KernelTables``): the same information re-laid for the fused CUDA
   residual.  Cell data are slot-major (``[slot][cell]``) so that a warp reading slot k of 32
   consecutive cells issues one coalesced 128-byte load; indices are int32; values that the
   reference derives on the fly from host-side constants (``1/d``, ``X_orthog``, limiter ``eps``,
   boundary offsets) are precomputed here with the reference's own operation order.

Quirk kept on purpose: the reference indexes the *flattened* list of Neumann values by component
number (``facet_boundary.py:278``, ``facet_process.py:192``).  All shipped configurations use zero
Neumann values, where this is harmless; the tables reproduce it exactly.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .config import BCMode, ConfigFVM


# ---------------------------------------------------------------------------------------------
# Sparse helpers (restated: ``sparse.py:231-325``, ``ell_kernel.py:225-256``)
# ---------------------------------------------------------------------------------------------
def lift_sparse_matrix(A_old: torch.Tensor, n_comp: int) -> torch.Tensor:
    """[M, N] -> [M*C, N*C] block-diagonal lift: entry (i, j) -> (i*C + c, j*C + c)."""
    A_old = A_old.coalesce()
    idx, val = A_old.indices(), A_old.values()
    M, N = A_old.size()
    comp = torch.arange(n_comp)
    rows = (idx[0].unsqueeze(1) * n_comp + comp.unsqueeze(0)).reshape(-1)
    cols = (idx[1].unsqueeze(1) * n_comp + comp.unsqueeze(0)).reshape(-1)
    vals = val.unsqueeze(1).expand(val.size(0), n_comp).reshape(-1)
    return torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (M * n_comp, N * n_comp)).coalesce()


def interleave_sparse_rows(tensors: list) -> torch.Tensor:
    """Stack k [m, n] COO matrices into [k*m, n] with row r of matrix i at k*r + i."""
    k = len(tensors)
    m, n = tensors[0].shape
    inds, vals = [], []
    for i, t in enumerate(tensors):
        t = t.coalesce()
        ind = t.indices().clone()
        ind[0] = k * ind[0] + i
        inds.append(ind)
        vals.append(t.values())
    return torch.sparse_coo_tensor(torch.cat(inds, 1), torch.cat(vals), (k * m, n)).coalesce()


def combine_facet_operators(A_main, A_bc, b_bc, bc_edge_mask, n_edges, n_cells, n_comp):
    """Merge interior-facet and boundary-facet operators into one [F*C, N*C] operator."""
    main_g = torch.where(~bc_edge_mask)[0]
    bc_g = torch.where(bc_edge_mask)[0]
    Ai, Av = A_main._indices(), A_main._values()
    Bi, Bv = A_bc._indices(), A_bc._values()
    rows_m = main_g[Ai[0] // n_comp] * n_comp + Ai[0] % n_comp
    rows_b = bc_g[Bi[0] // n_comp] * n_comp + Bi[0] % n_comp
    A_all = torch.sparse_coo_tensor(
        torch.stack([torch.cat([rows_m, rows_b]), torch.cat([Ai[1], Bi[1]])]),
        torch.cat([Av, Bv]), (n_edges * n_comp, n_cells * n_comp), dtype=A_main.dtype).coalesce()
    b_all = torch.zeros(n_edges * n_comp, dtype=b_bc.dtype)
    r = torch.arange(b_bc.numel())
    b_all[bc_g[r // n_comp] * n_comp + r % n_comp] = b_bc
    return A_all, b_all


def coo_to_ell(A: torch.Tensor, K: int | None = None):
    """Row-major ELL (vals [M, K], cols [M, K] int64) of a COO/CSR matrix.

    Same packing as ``csr_to_ell``: slot k of row r holds the k-th entry of the row in ascending
    column order; padded slots are col 0 / val 0; ``ValueError`` if a row exceeds ``K``.
    """
    if A.layout != torch.sparse_csr:
        A = A.coalesce().to_sparse_csr()
    crow, col, val = A.crow_indices(), A.col_indices(), A.values()
    M = A.shape[0]
    nnz = crow[1:] - crow[:-1]
    if K is None:
        K = int(nnz.max().item()) if M > 0 and nnz.numel() else 0
    if torch.any(nnz > K):
        raise ValueError("Some rows have more nonzeros than K")
    ell_c = torch.zeros((M, K), dtype=col.dtype)
    ell_v = torch.zeros((M, K), dtype=val.dtype)
    for k in range(K):
        rows = torch.nonzero(nnz > k, as_tuple=False).flatten()
        src = crow[rows] + k
        ell_c[rows, k] = col[src]
        ell_v[rows, k] = val[src]
    return ell_v, ell_c


# ---------------------------------------------------------------------------------------------
# Boundary specification
# ---------------------------------------------------------------------------------------------
@dataclass
class BCSpec:
    dirich_mask: torch.Tensor     # [Fb, C] bool
    neumann_mask: torch.Tensor    # [Fb, C] bool
    dirich_val: torch.Tensor      # flattened masked values (reference layout)
    neumann_val: torch.Tensor     # flattened masked values (reference layout)
    farfield_mask: torch.Tensor   # [Fb] bool
    inlet_mask: torch.Tensor      # [Fb] bool


def bc_spec_from_tags(bc_tags: dict, n_bc: int) -> BCSpec:
    """``FacetCalc._init_bc`` (``facet_process.py:297-330``) without the device side effects."""
    dm, nm, dv, nv, ff, il = [], [], [], [], [], []
    for _, e in bc_tags.items():
        dm.append(e.dirichlet())
        nm.append(e.neumann())
        dv.append(e.U)
        nv.append(e.dUdn)
        ff.append(e.farfield())
        il.append(e.inlet())
    if n_bc == 0:
        z = torch.zeros((0, 0), dtype=torch.bool)
        return BCSpec(z, z, torch.zeros(0), torch.zeros(0), torch.zeros(0, dtype=torch.bool),
                      torch.zeros(0, dtype=torch.bool))
    dirich_mask, neumann_mask = torch.tensor(dm), torch.tensor(nm)
    dvt = torch.tensor(dv, dtype=torch.float32)
    nvt = torch.tensor(nv, dtype=torch.float32)
    spec = BCSpec(dirich_mask, neumann_mask, dvt[dirich_mask], nvt[neumann_mask],
                  torch.tensor(ff), torch.tensor(il))
    assert spec.dirich_mask.shape[0] == n_bc, "Wrong mask shape"
    assert spec.farfield_mask.shape[0] == n_bc, "Wrong mask shape"
    return spec


@dataclass
class CharGroup:
    """A merged characteristic BC group (``facet_boundary.py:64-80``, ``BC.__init__`` ``:289-385``)."""
    bc_idx: torch.Tensor      # [Fc] boundary-local facet indices (sorted)
    cells: torch.Tensor       # [Fc] adjacent cells
    normals: torch.Tensor     # [Fc, dim] outward unit normals
    rho_inf: torch.Tensor
    v_n_inf: torch.Tensor     # outward-positive
    v_t_inf: torch.Tensor     # [Fc, dim]
    p_inf: torch.Tensor


@dataclass
class ReferenceOperators:
    G_mats: torch.Tensor            # COO [dim*N, N+Fb] (interleaved rows)
    flux_mat: torch.Tensor          # COO [N, F]
    A_face_grad: torch.Tensor       # COO [F*C, N*C]
    b_face_grad: torch.Tensor       # [F*C]
    A_bc: torch.Tensor | None       # COO [Fb*C, N*C]
    b_bc: torch.Tensor | None       # [Fb*C]
    A_corr: torch.Tensor | None     # COO [Fb*C, N*dim*C]


@dataclass
class KernelTables:
    """Flat arrays consumed by the CUDA residual (host copies; ``to(device)`` uploads them)."""
    dim: int
    n_comp: int
    n_cells: int
    n_facets: int
    n_bc: int
    n_char: int
    kg: int
    kf: int
    # cells
    g_vals: torch.Tensor      # [dim, kg, N] f32
    g_cols: torch.Tensor      # [kg, N] i32 (index into [prims; boundary facet values])
    nb_slot: torch.Tensor     # [N] i32: 4 bits per local facet j -> slot of its neighbour in g_cols
    disp: torch.Tensor        # [K, dim, N] f32 centroid -> facet midpoint
    eps: torch.Tensor         # [N] f32 limiter epsilon
    c2f: torch.Tensor         # [K, N] i32 cell -> facet
    side: torch.Tensor        # [N] i32 bit j = side (0 left, 1 right) of local facet j
    f_vals: torch.Tensor      # [kf, N] f32 divergence weights (+-1/vol)
    f_cols: torch.Tensor      # [kf, N] i32 facet indices
    inv_h: torch.Tensor       # [N] f64 max facet area / volume (CFL length scale inverse)
    volumes: torch.Tensor     # [N] f64
    centroids: torch.Tensor   # [N, dim] f32 (host only: corrector features)
    # facets
    fcell: torch.Tensor       # [F, 2] i32 (side 0 cell, side 1 cell); boundary: the cell twice
    fbc: torch.Tensor         # [F] i32 boundary-local index or -1
    normals: torch.Tensor     # [F, dim] f32
    fsize: torch.Tensor       # [F] f32 |normal|
    xorth: torch.Tensor       # [F, dim] f32 non-orthogonal correction vector (0 on boundary)
    inv_d: torch.Tensor       # [F] f32 1 / projected centroid distance (interior)
    # boundary facets
    bc_face: torch.Tensor     # [Fb] i32
    bc_side: torch.Tensor     # [Fb] i32
    bc_cell: torch.Tensor     # [Fb] i32
    bc_kind: torch.Tensor     # [Fb, C] i32: 1 Dirichlet, 2 Neumann, 0 other
    bc_b: torch.Tensor        # [Fb, C] f32 offset of the face value (b_bc)
    bc_l: torch.Tensor        # [Fb, dim] f32 tangential lever arm (A_corr)
    bc_ga: torch.Tensor       # [Fb, C] f32 face-gradient coefficient on the cell value
    bc_gb: torch.Tensor       # [Fb, C] f32 face-gradient offset
    bc_char: torch.Tensor     # [Fb] i32 index into the characteristic arrays or -1
    ch_cell: torch.Tensor     # [Fc] i32 cell of each characteristic facet
    ch_normal: torch.Tensor   # [Fc, dim] f32
    ch_rho: torch.Tensor      # [Fc] f32
    ch_vn: torch.Tensor       # [Fc] f32
    ch_vt: torch.Tensor       # [Fc, dim] f32
    ch_p: torch.Tensor        # [Fc] f32

    def to(self, device) -> "KernelTables":
        out = {}
        for k, v in self.__dict__.items():
            out[k] = v.contiguous().to(device) if isinstance(v, torch.Tensor) else v
        return KernelTables(**out)

    def records(self) -> dict:
        """The device record layout of ``include/fvm_b200.h`` (cell, divergence and facet records).

        Cell record [N][CR]: for the reference's stencil (compact, CR = 20 / 32) the KG - 1
        neighbour columns in slot order (int32 bits, the own slot in bits 28..30 of the first;
        padded to four), G weights [dim][KG], centroid->facet displacements [K][dim], limiter
        epsilon; for a widened stencil G weights [dim][KG], G columns [KG], displacements,
        epsilon, meta (int32 bits), zero padding.
        Divergence record [N][8]: weights [kf], facet indices [kf] (int32 bits), padding.
        Facet record [F][FR]: side-0 cell, side-1 cell (int32 bits; a boundary side holds
        -1 - boundary index), +-1/d (negative: side 1's cell has the lower index), |S|, normal [dim],
        non-orthogonal vector [dim], side-0 and
        side-1 centroid->facet displacements [dim] each, padding.
        """
        dim, N, F, K, kg, kf = self.dim, self.n_cells, self.n_facets, self.dim + 1, self.kg, self.kf
        CR, FR, DR = record_sizes(dim, kg)
        bits = lambda t: t.to(torch.int32).view(torch.float32)
        cell = torch.zeros((N, CR), dtype=torch.float32)
        weights = self.g_vals.permute(2, 0, 1).reshape(N, dim * kg)
        if kg == dim + 1 + 1:
            # compact record (the reference's stencil: every slot valid, the cell itself in one of
            # them): the kg - 1 neighbour columns in slot order, the own slot in the top bits of the
            # first; no meta word
            cols = self.g_cols.t().long()                                   # [N, kg]
            own = torch.arange(N).unsqueeze(1)
            is_self = cols == own
            one = is_self.sum(1) == 1
            # rows without their own column are never updated (a partition's halo copies, whose
            # stencil is left empty): they keep their first kg - 1 columns and the last slot
            empty = (self.g_vals == 0).all(dim=0).all(dim=0)
            assert bool((one | empty).all()), "gradient row without exactly one own column"
            assert N + self.n_bc < (1 << SELF_SLOT_SHIFT), "mesh too large for the compact cell record"
            is_self = torch.where(one.unsqueeze(1), is_self, torch.arange(kg).unsqueeze(0) == kg - 1)
            slot = is_self.int().argmax(1)
            nbr = cols[~is_self].view(N, kg - 1)
            nbr[:, 0] |= slot.long() << SELF_SLOT_SHIFT
            cell[:, 0:kg - 1] = bits(nbr.to(torch.int32))    # one 128-bit load (padded to 4 slots)
            o = 4
            cell[:, o:o + dim * kg] = weights
            o += dim * kg
            cell[:, o:o + K * dim] = self.disp.permute(2, 0, 1).reshape(N, K * dim)
            o += K * dim
            cell[:, o] = self.eps
        else:
            cell[:, 0:dim * kg] = weights
            o = dim * kg
            cell[:, o:o + kg] = bits(self.g_cols.t().contiguous())
            o += kg
            cell[:, o:o + K * dim] = self.disp.permute(2, 0, 1).reshape(N, K * dim)
            o += K * dim
            cell[:, o] = self.eps
            cell[:, o + 1] = bits(self.nb_slot)
        div = torch.zeros((N, DR), dtype=torch.float32)
        div[:, :kf] = self.f_vals.t()
        div[:, K:K + kf] = bits(self.f_cols.t().contiguous())
        # per facet side: centroid -> facet displacement of the cell on that side
        fdisp = torch.zeros((F, 2, dim), dtype=torch.float32)
        for j in range(K):
            fdisp[self.c2f[j].long(), ((self.side >> j) & 1).long()] = self.disp[j].t()
        codes = self.fcell.clone()
        if self.n_bc:
            b = torch.arange(self.n_bc, dtype=torch.int32)
            codes[self.bc_face.long(), self.bc_side.long()] = -1 - b
        face = torch.zeros((F, FR), dtype=torch.float32)
        face[:, 0] = bits(codes[:, 0].contiguous())
        face[:, 1] = bits(codes[:, 1].contiguous())
        # 1/d, negative when the side-1 cell precedes the side-0 cell in the cell numbering (the
        # order in which the facet's normal-gradient row sums its two terms)
        order = torch.where(self.fcell[:, 0] < self.fcell[:, 1], 1.0, -1.0).to(torch.float32)
        face[:, 2] = self.inv_d * order
        face[:, 3] = self.fsize
        face[:, 4:4 + dim] = self.normals
        face[:, 4 + dim:4 + 2 * dim] = self.xorth
        face[:, 4 + 2 * dim:4 + 3 * dim] = fdisp[:, 0]
        face[:, 4 + 3 * dim:4 + 4 * dim] = fdisp[:, 1]
        return dict(cell_rec=cell, div_rec=div, face_rec=face)


def record_sizes(dim: int, kg: int | None = None):
    """(cell record, facet record, divergence record) widths in floats.  The reference's stencil
    (kg = dim + 2) has the compact cell record FVM_CELL_REC(dim) (20 / 32); a widened stencil the
    generic one FVM_CELL_REC_KG(dim, kg) (kg slots and a meta word, padded to 8 floats)."""
    if kg is None or kg == dim + 2:
        return ((20 if dim == 2 else 32), 16, 8)
    return ((dim * kg + kg + (dim + 1) * dim + 2 + 7) // 8 * 8, 16, 8)


SELF_SLOT_SHIFT = 28     # compact cell record: bits 28..30 of the first column word = the cell's own slot


def row_sizes(dim: int):
    """(padded state row, limited-gradient row) widths in floats (FVM_ROW, FVM_GROW)."""
    return (4, 8) if dim == 2 else (8, 16)


def grad_index(dim: int, d: int, comp: int) -> int:
    """Position of d(comp)/dx_d in a limited-gradient row (V_k and T per direction, rho last)."""
    if comp == dim:
        return dim * (dim + 1) + d
    return d * (dim + 1) + (comp if comp < dim else dim)


# ---------------------------------------------------------------------------------------------
# Assembly
# ---------------------------------------------------------------------------------------------
class FVMTables:
    """Host assembly of everything ``FacetCalc``/``MeshCache``/``BoundarySetter`` precompute.

    ``mesh`` is a ``fvm_mesh.FVMMesh2D/3D``; ``bc_tags`` maps boundary-facet index -> ``Facet``.
    """

    def __init__(self, mesh, cfg: ConfigFVM, n_comp: int, bc_tags: dict, phy=None):
        self.mesh = mesh
        self.cfg = cfg
        self.dim = dim = mesh.dim
        self.n_comp = C = n_comp
        self.K = K = dim + 1
        self.n_cells = N = mesh.n_cells
        self.n_facets = F = mesh.n_facets
        self.bc_mask = mesh.bc_facet_mask
        self.n_bc = Fb = int(self.bc_mask.sum().item())
        R = cfg.C_v * (cfg.gamma - 1)
        self.R, self.gamma = R, cfg.gamma

        # --- MeshCache (facet_process.py:58-105) ---
        self.cent_to_facet_disp = mesh.cent_to_facet_disp.unsqueeze(-1)
        self.cell_facet_signs = (-mesh.cell_facet_signs + 1 / 2).to(torch.int32).view(K * N)
        self.cell_to_facet = mesh.cell_to_facet.view(K * N)
        cell_disps, facet_dists_bc, _, neigh_combine = mesh.cell_grad_stuff
        self.facet_dists_bc = facet_dists_bc.unsqueeze(-1).expand(-1, C)
        self.neigh_combine = neigh_combine
        self.normals = mesh.normals
        self.facet_size = torch.norm(self.normals, dim=1, keepdim=True)
        normal_hat = self.normals / self.facet_size
        self.normals_hat = normal_hat.unsqueeze(-1)
        cdf = torch.full((F, dim), float("nan"))
        cdf[~self.bc_mask] = cell_disps
        d_cos_theta = (normal_hat * cdf).sum(dim=1)
        self.cell_dist_proj = d_cos_theta
        X_orthog = cdf / d_cos_theta.unsqueeze(-1) - normal_hat
        X_orthog[self.bc_mask] = 0
        self.X_orthog = X_orthog
        face_assigned = torch.zeros((F, max(dim, 2)), dtype=torch.bool)
        face_assigned[self.cell_to_facet, self.cell_facet_signs] = True
        assigned_boundary = face_assigned[self.bc_mask]
        self.bc_facet_side = (~assigned_boundary).float().argmax(dim=1).int()
        self.bc_locations = torch.where(self.bc_mask)[0].int()
        self.facet_to_cell_bc = mesh.facet_to_cell_bc.reshape(-1)
        self.facet_to_cell_main = mesh.facet_to_cell_main

        # Slope limiter epsilon (limiter.py:9-14)
        areas = mesh.volumes.view(-1, 1, 1)
        self.eps_p = (cfg.lim_K * areas ** 0.5) ** (cfg.lim_p + 1)

        # --- Boundary specification (facet_process.py:297-330) ---
        self.bc = bc_spec_from_tags(bc_tags, Fb)
        self.char_groups = self._build_char_groups() if Fb else {}

        self.ops = self._build_reference_operators()
        self.kernel = self._build_kernel_tables()

    # -- reference operators ------------------------------------------------------------------
    def _build_flux_mat(self):
        N, K = self.n_cells, self.K
        rows = torch.arange(N).unsqueeze(1).expand(N, K).reshape(-1)
        cols = self.cell_to_facet.reshape(-1)
        vals = self.cell_facet_signs.reshape(-1).to(torch.float32) * 2 - 1
        vinv = (1.0 / self.mesh.volumes).to(torch.float32)
        D = vals * vinv[rows]
        return torch.sparse_coo_tensor(torch.stack([rows, cols]), D, [N, self.n_facets],
                                       dtype=torch.float32).coalesce()

    def _build_face_grads(self):
        """``MeshCache.build_spm_face_grads`` (``facet_process.py:114-198``)."""
        C, N, Fb = self.n_comp, self.n_cells, self.n_bc
        fm = self.facet_to_cell_main
        nf = fm.shape[0]
        rows = torch.arange(nf).repeat_interleave(2)
        cols = fm.reshape(-1)
        rep = self.cell_dist_proj[~self.bc_mask].repeat_interleave(2)
        signs = torch.tensor([-1, 1], dtype=torch.float32).repeat(nf)
        vals = signs / rep
        A_main = lift_sparse_matrix(torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (nf, N)), C)
        if Fb == 0:
            A_bc = torch.sparse_coo_tensor(torch.zeros((2, 0), dtype=torch.long), torch.zeros(0), (0, N * C))
            return combine_facet_operators(A_main, A_bc.coalesce(), torch.zeros(0), self.bc_mask,
                                           self.n_facets, N, C)
        bc_rows = torch.arange(Fb).unsqueeze(1).expand(Fb, C).reshape(-1)
        comp_idx = torch.arange(C).unsqueeze(0).expand(Fb, C).reshape(-1)
        dir_rows = torch.nonzero(self.bc.dirich_mask.reshape(-1), as_tuple=False).squeeze(1)
        dir_f = bc_rows[dir_rows]
        neu_rows = torch.nonzero(self.bc.neumann_mask.reshape(-1), as_tuple=False).squeeze(1)
        neu_comp = comp_idx[neu_rows]
        gcols = self.facet_to_cell_bc[dir_f] * C + comp_idx[dir_rows]
        gvals = -1.0 / self.facet_dists_bc[dir_f, 0]
        A_grad_bc = torch.sparse_coo_tensor(torch.stack([dir_rows, gcols]), gvals, (Fb * C, N * C))
        b_grad = torch.zeros(Fb * C, dtype=torch.float32)
        b_grad[dir_rows] = self.bc.dirich_val / self.facet_dists_bc[dir_f, 0]
        b_grad[neu_rows] = self.bc.neumann_val[neu_comp]
        return combine_facet_operators(A_main, A_grad_bc, b_grad, self.bc_mask, self.n_facets, N, C)

    def _neumann_geometry(self):
        """Per Neumann (facet, comp) entry: cell, lever arm l = r - (r.n)n (``facet_boundary.py:82-115``)."""
        C, K, dim = self.n_comp, self.K, self.dim
        mask_all = torch.zeros((self.n_facets, C), dtype=torch.bool)
        mask_all[self.bc_mask] = self.bc.neumann_mask
        w_all = torch.where(mask_all)
        where_neum = torch.where(self.bc.neumann_mask)
        bc_f2c = torch.zeros(self.n_facets, dtype=torch.long)
        bc_f2c[self.bc_mask] = self.facet_to_cell_bc
        neum_cells = bc_f2c[w_all[0]]
        c2f = self.cell_to_facet.view(-1, K)
        hit = w_all[0].unsqueeze(-1).repeat(1, K) == c2f[neum_cells]
        cell_facet_id = torch.where(hit)[1]
        n_hats = self.normals_hat.squeeze(-1)[w_all[0]]
        ctf = self.cent_to_facet_disp[neum_cells].squeeze(-1)
        r = ctf[torch.arange(ctf.shape[0]), cell_facet_id]
        d = n_hats * (r * n_hats).sum(dim=1, keepdim=True)
        return where_neum, neum_cells, r - d

    def _build_bc_operators(self):
        C, N, Fb, dim = self.n_comp, self.n_cells, self.n_bc, self.dim
        nrows = Fb * C
        bc_rows = torch.arange(Fb).unsqueeze(1).expand(Fb, C).reshape(-1)
        comp_idx = torch.arange(C).unsqueeze(0).expand(Fb, C).reshape(-1)
        dmask = self.bc.dirich_mask.reshape(-1)
        nmask = self.bc.neumann_mask.reshape(-1)
        ni = torch.nonzero(nmask, as_tuple=False).squeeze(1)
        acols = self.facet_to_cell_bc[bc_rows[ni]] * C + comp_idx[ni]
        A_bc = torch.sparse_coo_tensor(torch.stack([ni, acols]), torch.ones_like(ni, dtype=torch.float32),
                                       (nrows, N * C)).coalesce()
        b_bc = torch.zeros(nrows, dtype=torch.float32)     # reference: torch.empty (never read)
        b_bc[dmask] = self.bc.dirich_val
        b_bc[nmask] = self.bc.neumann_val[comp_idx[nmask]] * self.facet_dists_bc.flatten()[nmask]

        where_neum, neum_cells, l = self._neumann_geometry()
        n_neum = neum_cells.shape[0]
        row_ids = where_neum[0] * C + where_neum[1]
        rows = row_ids[:, None].expand(n_neum, dim).reshape(-1)
        sp = torch.arange(dim)
        cols = (neum_cells[:, None] * (dim * C) + sp[None, :] * C + where_neum[1][:, None]).reshape(-1)
        A_corr = torch.sparse_coo_tensor(torch.stack([rows, cols]), l.reshape(-1),
                                         (nrows, N * dim * C)).coalesce()
        self._neum = (where_neum, neum_cells, l)
        return A_bc, b_bc, A_corr

    def _build_reference_operators(self) -> ReferenceOperators:
        G = interleave_sparse_rows([self.mesh.gradient_coo(d) for d in range(self.dim)])
        A_fg, b_fg = self._build_face_grads()
        if self.n_bc:
            A_bc, b_bc, A_corr = self._build_bc_operators()
        else:
            A_bc = b_bc = A_corr = None
        return ReferenceOperators(G, self._build_flux_mat(), A_fg, b_fg, A_bc, b_bc, A_corr)

    # -- characteristic groups -----------------------------------------------------------------
    def _build_char_groups(self):
        """Merged characteristic BC groups (``BoundarySetter.__init__`` ``facet_boundary.py:46-80``)."""
        cfg, dim = self.cfg, self.dim
        specs = {}
        nh = self.normals_hat.squeeze(-1)[self.bc_mask]
        for mask, bcfg in ((self.bc.farfield_mask, cfg.exit_cfg), (self.bc.inlet_mask, cfg.inlet_cfg)):
            if not bool(torch.any(mask)):
                continue
            sign = 2 * (self.bc_facet_side[mask] - 0.5)
            normals = nh[mask] * sign.unsqueeze(-1)
            specs.setdefault(bcfg.mode, []).append((bcfg, mask, self.facet_to_cell_bc[mask], normals))
        groups = {}
        for mode, sp in specs.items():
            # by name, so that the reference's own BCMode enum (a different class) is accepted too
            if getattr(mode, "name", None) != BCMode.Characteristic.name:
                raise NotImplementedError(
                    f"BCMode {mode} is not supported: only Characteristic boundaries are implemented "
                    "(the reference's Farfield mode cannot run: facet_boundary.py:607)")
            merged = sp[0][1].clone()
            for s in sp[1:]:
                merged = merged | s[1]
            bc_idx = torch.where(merged)[0]
            face_to_pos = torch.full((self.n_bc,), -1, dtype=torch.long)
            off = 0
            for s in sp:
                idx = torch.where(s[1])[0]
                face_to_pos[idx] = torch.arange(off, off + idx.shape[0])
                off += idx.shape[0]
            perm = face_to_pos[bc_idx]
            cat = lambda lst: torch.cat(lst)[perm]
            nl, rl, vnl, vtl, pl = [], [], [], [], []
            for bcfg, mask, cells, normals in sp:
                n = int(mask.sum().item())
                nl.append(normals)
                T_inf = torch.full((n,), float(bcfg.T_inf))
                rho_inf = torch.full((n,), float(bcfg.rho_inf))
                rl.append(rho_inf)
                if dim == 2:
                    tangents = torch.stack((-normals[:, 1], normals[:, 0]), dim=1)
                    vtl.append(tangents * bcfg.v_t_inf)
                    vnl.append(torch.full((n,), -float(bcfg.v_n_inf)))
                else:
                    v_inf = torch.tensor(bcfg.v_inf, dtype=torch.float32)
                    v_n = (normals * v_inf).sum(dim=1)
                    vtl.append(v_inf - normals * v_n.unsqueeze(-1))
                    vnl.append(v_n)
                pl.append(self.R * rho_inf * T_inf)
            cells = torch.cat([s[2] for s in sp])[perm]
            groups[mode] = CharGroup(bc_idx, cells, cat(nl), cat(rl), cat(vnl), cat(vtl), cat(pl))
        return groups

    # -- kernel tables -------------------------------------------------------------------------
    def _build_kernel_tables(self) -> KernelTables:
        dim, C, N, F, Fb, K = self.dim, self.n_comp, self.n_cells, self.n_facets, self.n_bc, self.K
        i32 = torch.int32
        # G: interleaved rows dim*i + d -> [dim, kg, N]
        gv, gc = coo_to_ell(self.ops.G_mats)
        kg = gv.shape[1]
        assert kg <= 16, "gradient stencil wider than 16"
        gv = gv.view(N, dim, kg)
        gc = gc.view(N, dim, kg)
        assert torch.equal(gc, gc[:, :1].expand_as(gc)), "gradient rows of one cell differ in columns"
        g_vals = gv.permute(1, 2, 0).contiguous()
        g_cols = gc[:, 0, :].t().contiguous().to(i32)
        # slot of neighbour j in the cell's G columns
        nb = self.neigh_combine.long()
        slot = (gc[:, 0, :].unsqueeze(1) == nb.unsqueeze(2)).int().argmax(dim=2)   # [N, K]
        assert torch.all((gc[:, 0, :].gather(1, slot) == nb)), "neighbour missing from G row"
        nb_slot = torch.zeros(N, dtype=torch.int64)
        for j in range(K):
            nb_slot |= slot[:, j].long() << (4 * j)
        # bits 24..28: number of valid (unpadded) slots of the cell's gradient row
        row_nnz = torch.bincount(self.ops.G_mats.coalesce().indices()[0], minlength=N * dim).view(N, dim)[:, 0]
        nb_slot |= row_nnz.long() << 24
        disp = self.mesh.cent_to_facet_disp.permute(1, 2, 0).contiguous()          # [K, dim, N]
        eps = self.eps_p.reshape(-1).contiguous()
        c2f = self.mesh.cell_to_facet.t().contiguous().to(i32)
        sides = self.cell_facet_signs.view(N, K).long()
        side = torch.zeros(N, dtype=torch.int64)
        for j in range(K):
            side |= sides[:, j] << j
        fv, fc = coo_to_ell(self.ops.flux_mat)
        kf = fv.shape[1]
        vol = self.mesh.volumes.double()
        amax = self.facet_size.squeeze(-1)[self.mesh.cell_to_facet].double().max(dim=1).values
        inv_h = amax / vol

        # facets
        fcell = torch.empty((F, 2), dtype=torch.int64)
        fcell[~self.bc_mask] = self.facet_to_cell_main
        bcc = self.facet_to_cell_bc
        fcell[self.bc_mask] = torch.stack([bcc, bcc], 1)
        fbc = torch.full((F,), -1, dtype=torch.int64)
        fbc[self.bc_mask] = torch.arange(Fb)
        inv_d = torch.zeros(F, dtype=torch.float32)
        inv_d[~self.bc_mask] = 1.0 / self.cell_dist_proj[~self.bc_mask]

        # boundary facets
        bc_kind = torch.zeros((Fb, C), dtype=i32)
        bc_b = torch.zeros((Fb, C), dtype=torch.float32)
        bc_l = torch.zeros((Fb, dim), dtype=torch.float32)
        bc_ga = torch.zeros((Fb, C), dtype=torch.float32)
        bc_gb = torch.zeros((Fb, C), dtype=torch.float32)
        bc_char = torch.full((Fb,), -1, dtype=i32)
        ch = None
        if Fb:
            bc_kind[self.bc.dirich_mask] = 1
            bc_kind[self.bc.neumann_mask] = 2
            bc_b = self.ops.b_bc.view(Fb, C).clone()
            wn, _, l = self._neum
            bc_l[wn[0]] = l
            # face-gradient rows of boundary facets, read back from the combined operator
            A = self.ops.A_face_grad.coalesce()
            rows, cols = A.indices()
            sel = self.bc_mask[rows // C]
            bl = torch.full((F,), -1, dtype=torch.long)
            bl[self.bc_mask] = torch.arange(Fb)
            rb = rows[sel]
            bc_ga.view(-1)[bl[rb // C] * C + rb % C] = A.values()[sel]
            bc_gb = self.ops.b_face_grad.view(F, C)[self.bc_mask].clone()
            if self.char_groups:
                (g,) = self.char_groups.values()
                bc_char[g.bc_idx] = torch.arange(g.bc_idx.shape[0], dtype=i32)
                ch = g
        if ch is None:
            z = torch.zeros(0, dtype=torch.float32)
            ch_n, ch_r, ch_vn, ch_vt, ch_p = torch.zeros((0, dim)), z, z, torch.zeros((0, dim)), z
            ch_cell = torch.zeros(0, dtype=i32)
            nchar = 0
        else:
            ch_n, ch_r, ch_vn, ch_vt, ch_p = ch.normals, ch.rho_inf, ch.v_n_inf, ch.v_t_inf, ch.p_inf
            ch_cell = ch.cells.to(i32)
            nchar = int(ch.bc_idx.shape[0])

        return KernelTables(
            dim=dim, n_comp=C, n_cells=N, n_facets=F, n_bc=Fb, n_char=nchar, kg=kg, kf=kf,
            g_vals=g_vals.float(), g_cols=g_cols, nb_slot=nb_slot.to(i32), disp=disp.float(),
            eps=eps.float(), c2f=c2f, side=side.to(i32),
            f_vals=fv.t().contiguous(), f_cols=fc.t().contiguous().to(i32),
            inv_h=inv_h, volumes=vol, centroids=self.mesh.centroids.float().contiguous(),
            fcell=fcell.to(i32), fbc=fbc.to(i32), normals=self.normals.contiguous(),
            fsize=self.facet_size.reshape(-1).contiguous(), xorth=self.X_orthog.contiguous(),
            inv_d=inv_d,
            bc_face=self.bc_locations.to(i32), bc_side=self.bc_facet_side.to(i32),
            bc_cell=self.facet_to_cell_bc.to(i32), bc_kind=bc_kind, bc_b=bc_b, bc_l=bc_l,
            bc_ga=bc_ga, bc_gb=bc_gb, bc_char=bc_char, ch_cell=ch_cell,
            ch_normal=ch_n.float().contiguous(), ch_rho=ch_r.float(), ch_vn=ch_vn.float(),
            ch_vt=ch_vt.float().contiguous(), ch_p=ch_p.float(),
        )
