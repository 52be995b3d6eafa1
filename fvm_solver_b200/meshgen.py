"""Synthetic mesh generators for the workloads (scipy Delaunay).

The reference meshes with gmsh (``mesh_gen/mesh_2d/create_mesh.py:60``,
``mesh_gen/mesh_3d/create_mesh.py:65``), which is not available here, so these generators stand in
for it.  They return meshes in the reference's input format
(``run_fvm.generate_mesh``, ``time_fvm/run_fvm.py:14-34``):

    vertices [V, dim] float32, cells [N, dim+1] int32, facets [F, dim] int64 (interior facets
    first, then boundary facets), bc_facet_mask [F] bool, boundary tags (one per boundary facet).

Cells, interior facets and boundary facets are each ordered along a Morton (Z-order) curve of
their centroids so that neighbouring cells sit close together in memory; this is what makes the
device-side neighbour gathers cache-friendly.  The ordering is a property of the generated mesh
itself (both the oracle and the CUDA path see the same numbering), not a hidden permutation.

``periodic_box`` builds a periodic tetrahedralisation (no boundary facets).  Each cell and facet
carries integer lattice shifts per vertex so that its unwrapped coordinates are
``vertices[idx] + shift * L``; ``fvm_mesh.FVMMesh3D`` consumes them.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch
from scipy.spatial import Delaunay


# ---------------------------------------------------------------------------------------------
# Morton ordering
# ---------------------------------------------------------------------------------------------
def _spread_bits(x: np.ndarray, dim: int) -> np.ndarray:
    x = x.astype(np.uint64)
    out = np.zeros_like(x)
    nbits = 21 if dim == 3 else 31
    for b in range(nbits):
        out |= ((x >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * dim)
    return out


def morton_order(points: np.ndarray) -> np.ndarray:
    """Permutation that sorts ``points`` [n, dim] along a Z-order curve."""
    dim = points.shape[1]
    lo = points.min(axis=0)
    span = np.maximum(points.max(axis=0) - lo, 1e-30)
    nb = 20 if dim == 3 else 30
    q = np.clip(((points - lo) / span * ((1 << nb) - 1)).astype(np.int64), 0, (1 << nb) - 1)
    key = np.zeros(len(points), dtype=np.uint64)
    for d in range(dim):
        key |= _spread_bits(q[:, d], dim) << np.uint64(d)
    return np.argsort(key, kind="stable")


@dataclass
class MeshSpec:
    """A generated mesh in the reference's input format (plus periodic shifts when periodic)."""
    vertices: torch.Tensor          # [V, dim] float32
    cells: torch.Tensor             # [N, dim+1] int32
    facets: torch.Tensor            # [F, dim] int64
    bc_facet_mask: torch.Tensor     # [F] bool
    bc_tags: list                   # [F_b] str, one per boundary facet in facet order
    bound_facets: torch.Tensor      # [F_b, dim] int64
    period: np.ndarray | None = None        # [dim] box lengths when periodic
    cell_shifts: torch.Tensor | None = None   # [N, dim+1, dim] int8
    facet_shifts: torch.Tensor | None = None  # [F, dim, dim] int8
    info: dict = field(default_factory=dict)

    @property
    def dim(self) -> int:
        return int(self.vertices.shape[1])

    @property
    def n_cells(self) -> int:
        return int(self.cells.shape[0])


def _facets_of_cells(cells: np.ndarray) -> np.ndarray:
    """All local facets [N, dim+1, dim] in the reference's local order.

    2D: (v0,v1), (v1,v2), (v2,v0) (``fvm_mesh.py:211-222``);
    3D: (0,1,2), (0,2,3), (0,3,1), (1,3,2) (``fvm_mesh.py:452-457``).
    """
    if cells.shape[1] == 3:
        pats = [(0, 1), (1, 2), (2, 0)]
    else:
        pats = [(0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 3, 2)]
    return np.stack([cells[:, list(p)] for p in pats], axis=1)


def _finish_mesh(pts: np.ndarray, tri: np.ndarray, tag_fn) -> MeshSpec:
    """Order cells/facets along a Morton curve, split interior / boundary facets and tag."""
    dim = pts.shape[1]
    cent = pts[tri].mean(axis=1)
    tri = tri[morton_order(cent)]
    loc = _facets_of_cells(tri).reshape(-1, dim)
    key = np.sort(loc, axis=1)
    uniq, counts = np.unique(key, axis=0, return_counts=True)
    assert counts.max() <= 2, "non-manifold facet"
    int_f, bnd_f = uniq[counts == 2], uniq[counts == 1]
    int_f = int_f[morton_order(pts[int_f].mean(axis=1))]
    bnd_f = bnd_f[morton_order(pts[bnd_f].mean(axis=1))]
    tags = [tag_fn(pts[f]) for f in bnd_f]
    facets = np.concatenate([int_f, bnd_f], axis=0)
    mask = np.concatenate([np.zeros(len(int_f), bool), np.ones(len(bnd_f), bool)])
    return MeshSpec(
        vertices=torch.from_numpy(pts.astype(np.float32)),
        cells=torch.from_numpy(tri.astype(np.int32)),
        facets=torch.from_numpy(facets.astype(np.int64)),
        bc_facet_mask=torch.from_numpy(mask),
        bc_tags=tags,
        bound_facets=torch.from_numpy(bnd_f.astype(np.int64)),
    )


def _drop_degenerate(pts: np.ndarray, tri: np.ndarray, tol: float) -> np.ndarray:
    p = pts[tri]
    if pts.shape[1] == 2:
        ab, ac = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]
        vol = 0.5 * np.abs(ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0])
    else:
        ab, ac, ad = p[:, 1] - p[:, 0], p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]
        vol = np.abs(np.einsum("ij,ij->i", ab, np.cross(ac, ad))) / 6.0
    return tri[vol > tol]


# ---------------------------------------------------------------------------------------------
# 2D channel with a circular cylinder
# ---------------------------------------------------------------------------------------------
def channel_cylinder(h: float = 0.02, radius: float = 0.1, center=(0.5, 0.5), length: float = 2.0,
                     height: float = 1.0, seed: int = 0, jitter: float = 0.1,
                     cylinder: bool = True) -> MeshSpec:
    """Channel [0, length] x [0, height] around a cylinder, target edge length ``h``.

    Boundary tags follow ``gen_rand_mesh`` (``mesh_gen/mesh_2d/meshes_fvm.py:88-94``):
    x = 0 -> "Left", x = length -> "Right", walls and the cylinder -> "NavierWall".
    """
    rng = np.random.default_rng(seed)
    nx, ny = max(2, int(round(length / h))), max(2, int(round(height / h)))
    xb, yb = np.linspace(0.0, length, nx + 1), np.linspace(0.0, height, ny + 1)
    bnd = [np.stack([xb, np.zeros_like(xb)], 1), np.stack([xb, np.full_like(xb, height)], 1),
           np.stack([np.zeros(ny - 1), yb[1:-1]], 1), np.stack([np.full(ny - 1, length), yb[1:-1]], 1)]
    cx, cy = center
    if cylinder:
        nc = max(12, int(round(2 * np.pi * radius / h)))
        th = 2 * np.pi * np.arange(nc) / nc
        bnd.append(np.stack([cx + radius * np.cos(th), cy + radius * np.sin(th)], 1))
    dy = h * np.sqrt(3.0) / 2.0
    rows = []
    for j, y in enumerate(np.arange(dy / 2, height, dy)):
        xs = np.arange(h / 2 if j % 2 else h, length, h)
        rows.append(np.stack([xs, np.full_like(xs, y)], 1))
    inner = np.concatenate(rows)
    inner = inner + rng.uniform(-jitter * h, jitter * h, inner.shape)
    keep = (np.minimum.reduce([inner[:, 0], length - inner[:, 0], inner[:, 1], height - inner[:, 1]])
            > 0.45 * h)
    if cylinder:
        keep &= np.hypot(inner[:, 0] - cx, inner[:, 1] - cy) > radius + 0.45 * h
    pts = np.concatenate(bnd + [inner[keep]])
    pts = pts[morton_order(pts)]
    tri = Delaunay(pts).simplices.astype(np.int64)
    if cylinder:
        c = pts[tri].mean(axis=1)
        tri = tri[np.hypot(c[:, 0] - cx, c[:, 1] - cy) > radius]
    tri = _drop_degenerate(pts, tri, 1e-14)

    def tag(fp):
        if np.all(np.abs(fp[:, 0]) < 1e-9):
            return "Left"
        if np.all(np.abs(fp[:, 0] - length) < 1e-9):
            return "Right"
        on_rect = np.all((np.abs(fp[:, 1]) < 1e-9) | (np.abs(fp[:, 1] - height) < 1e-9))
        on_cyl = cylinder and np.all(np.abs(np.hypot(fp[:, 0] - cx, fp[:, 1] - cy) - radius) < 1e-6)
        assert on_rect or on_cyl, f"stray boundary facet {fp}"
        return "NavierWall"

    spec = _finish_mesh(pts, tri, tag)
    spec.info = dict(kind="channel_cylinder", h=h, radius=radius, center=tuple(center), seed=seed)
    return spec


def channel_cylinder_cells(n_cells: int, **kw) -> MeshSpec:
    """Channel-cylinder mesh with approximately ``n_cells`` triangles."""
    length, height, radius = kw.get("length", 2.0), kw.get("height", 1.0), kw.get("radius", 0.1)
    area = length * height - np.pi * radius ** 2
    h = float(np.sqrt(area / (n_cells * np.sqrt(3.0) / 4.0)))
    return channel_cylinder(h=h, **kw)


# ---------------------------------------------------------------------------------------------
# 3D flow over a sphere
# ---------------------------------------------------------------------------------------------
def sphere_box(n_cells: int = 500_000, radius: float = 0.5, box=((-5.0, 15.0), (-5.0, 5.0), (-5.0, 5.0)),
               seed: int = 0, jitter: float = 0.2, levels: int = 4) -> MeshSpec:
    """Tetrahedral mesh of a box around a sphere at the origin, with about ``n_cells`` tets.

    Points are nested jittered grids: spacing H over the whole box and H / 2^l inside boxes around
    the sphere that shrink with the level l (finest next to the sphere), each level's grid cut out
    of the coarser ones; grid points on the box faces stay on their planes, and a Fibonacci lattice
    at the finest spacing lies on the sphere.  After the Delaunay tetrahedralisation, tets whose
    centroid lies inside the sphere are removed.  Boundary tags: the sphere "NavierWall", the
    x-min face "Left" (inlet), the x-max face "Right" (exit), the four side faces "Farfield".
    """
    rng = np.random.default_rng(seed)
    lo = np.array([b[0] for b in box], dtype=np.float64)
    hi = np.array([b[1] for b in box], dtype=np.float64)
    ext = hi - lo

    def grid(a, b, h, on_faces):
        n = np.maximum(1, np.round((b - a) / h).astype(int))
        axes = [np.linspace(a[d], b[d], n[d] + 1) for d in range(3)]
        P = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
        hh = (b - a) / n
        on = np.zeros_like(P, dtype=bool)
        if on_faces:
            on = (np.abs(P - lo) < 1e-9) | (np.abs(P - hi) < 1e-9)
        return P + np.where(on, 0.0, rng.uniform(-jitter, jitter, P.shape) * hh), hh.min()

    # level boxes: level l covers [-w_l, w_l]^3 around the sphere (clipped to the domain), w_l shrinking
    def level_box(l):
        w = radius * 2.5 * 2.0 ** (levels - 1 - l)
        return np.maximum(lo, -w), np.minimum(hi, w)

    def count(H):
        tot = np.prod(ext / H)
        for l in range(1, levels):
            a, b = level_box(l)
            tot += np.prod((b - a) / (H / 2 ** l)) * (1 - 1 / 8)
        return tot * 7.0                      # ~7 tets per grid point (measured)

    H = float(ext.min() / 8)
    for _ in range(60):                       # spacing for the requested cell count
        H *= (count(H) / n_cells) ** (1 / 3)
    pts, _ = grid(lo, hi, H, True)
    for l in range(1, levels):
        a, b = level_box(l)
        h = H / 2 ** l
        inside = np.all((pts > a + 1e-9) & (pts < b - 1e-9), axis=1)
        pts = pts[~inside]
        fine, _ = grid(a, b, h, True)
        keep = np.all((fine > a - 1e-9) & (fine < b + 1e-9), axis=1)
        pts = np.concatenate([pts, fine[keep]])
    h_min = H / 2 ** (levels - 1)
    # points near the sphere: remove those inside or too close, add a surface lattice
    r = np.linalg.norm(pts, axis=1)
    pts = pts[r > radius + 0.45 * h_min]
    n_s = max(60, int(round(4 * np.pi * radius ** 2 / (h_min ** 2 * np.sqrt(3) / 2))))
    k = np.arange(n_s) + 0.5
    phi = np.arccos(1 - 2 * k / n_s)
    th = np.pi * (1 + 5 ** 0.5) * k
    surf = radius * np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], 1)
    pts = np.unique(np.round(np.concatenate([pts, surf]), 12), axis=0)
    pts = pts[morton_order(pts)]
    tet = Delaunay(pts).simplices.astype(np.int64)
    c = pts[tet].mean(axis=1)
    tet = tet[np.linalg.norm(c, axis=1) > radius]
    tet = _drop_degenerate(pts, tet, 1e-14 * float(np.prod(ext)) / len(pts))

    def tag(fp):
        if np.all(np.abs(np.linalg.norm(fp, axis=1) - radius) < 1e-6):
            return "NavierWall"
        if np.all(np.abs(fp[:, 0] - lo[0]) < 1e-9):
            return "Left"
        if np.all(np.abs(fp[:, 0] - hi[0]) < 1e-9):
            return "Right"
        on_side = any(np.all(np.abs(fp[:, d] - v) < 1e-9) for d in (1, 2) for v in (lo[d], hi[d]))
        assert on_side, f"stray boundary facet {fp}"
        return "Farfield"

    spec = _finish_mesh(pts, tet, tag)
    spec.info = dict(kind="sphere_box", radius=radius, seed=seed, spacing=H, spacing_min=h_min)
    return spec


# ---------------------------------------------------------------------------------------------
# 3D boxes
# ---------------------------------------------------------------------------------------------
def box3d(n: int = 12, size: float = 1.0, seed: int = 0, jitter: float = 0.2,
          inlet_axis: int = 0) -> MeshSpec:
    """Non-periodic jittered-grid tetrahedral box [0, size]^3.

    Facets on the two ``inlet_axis`` ends are tagged "Farfield" (the reference's 3D setup maps that
    tag to a characteristic inlet, ``run_fvm_3d.py:44-45``); the other four sides "NavierWall".
    Boundary points stay on their planes so the Delaunay hull is the box.
    """
    rng = np.random.default_rng(seed)
    h = size / n
    g = np.arange(n + 1) * h
    P = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    on = (np.abs(P) < 1e-12) | (np.abs(P - size) < 1e-12)
    P = P + np.where(on, 0.0, rng.uniform(-jitter * h, jitter * h, P.shape))
    P = P[morton_order(P)]
    tet = _drop_degenerate(P, Delaunay(P).simplices.astype(np.int64), 1e-14 * size ** 3)

    def tag(fp):
        if np.all(np.abs(fp[:, inlet_axis]) < 1e-9) or np.all(np.abs(fp[:, inlet_axis] - size) < 1e-9):
            return "Farfield"
        return "NavierWall"

    spec = _finish_mesh(P, tet, tag)
    spec.info = dict(kind="box3d", n=n, size=size, seed=seed)
    return spec


def periodic_box(n: int = 70, length: float = 2 * np.pi, seed: int = 0, jitter: float = 0.2,
                 margin: float = 2.5) -> MeshSpec:
    """Periodic jittered-grid Delaunay tetrahedralisation of [0, length)^3.

    ``n`` points per axis (spacing h = length / n), jitter ``jitter * h`` per coordinate.  The
    point set is extended by its periodic images within ``margin * h`` of the box, triangulated, and
    the tetrahedra whose centroid lies in the fundamental box are kept: every periodic class of
    tetrahedra has exactly one such representative.  All facets are interior (F = 2N).
    """
    rng = np.random.default_rng(seed)
    h = length / n
    g = (np.arange(n) + 0.5) * h
    P = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    P = np.mod(P + rng.uniform(-jitter * h, jitter * h, P.shape), length)
    P = P[morton_order(P)]
    m = margin * h
    ext_pts, ext_idx, ext_sh = [P], [np.arange(len(P))], [np.zeros((len(P), 3), np.int8)]
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            for sz in (-1, 0, 1):
                if sx == sy == sz == 0:
                    continue
                s = np.array([sx, sy, sz])
                Q = P + s * length
                sel = np.all((Q > -m) & (Q < length + m), axis=1)
                ext_pts.append(Q[sel])
                ext_idx.append(np.nonzero(sel)[0])
                ext_sh.append(np.broadcast_to(s.astype(np.int8), (int(sel.sum()), 3)))
    EP = np.concatenate(ext_pts)
    EI = np.concatenate(ext_idx)
    ES = np.concatenate(ext_sh)
    tet = Delaunay(EP).simplices.astype(np.int64)
    cen = EP[tet].mean(axis=1)
    tet = tet[np.all((cen >= 0) & (cen < length), axis=1)]
    tet = _drop_degenerate(EP, tet, 1e-12 * h ** 3)
    cen = EP[tet].mean(axis=1)
    tet = tet[morton_order(cen)]
    cells = EI[tet]                                   # [N, 4] fundamental vertex ids
    cshift = ES[tet]                                  # [N, 4, 3] lattice shifts
    vol = np.abs(np.einsum("ij,ij->i", EP[tet[:, 1]] - EP[tet[:, 0]],
                           np.cross(EP[tet[:, 2]] - EP[tet[:, 0]], EP[tet[:, 3]] - EP[tet[:, 0]]))) / 6
    assert abs(vol.sum() - length ** 3) < 1e-6 * length ** 3, f"periodic volume {vol.sum()} != {length ** 3}"

    # Facets: key = (sorted vertex ids, lattice shifts relative to the smallest-id vertex).
    pats = [(0, 1, 2), (0, 2, 3), (0, 3, 1), (1, 3, 2)]
    lv = np.stack([cells[:, list(p)] for p in pats], 1).reshape(-1, 3)
    ls = np.stack([cshift[:, list(p)] for p in pats], 1).reshape(-1, 3, 3).astype(np.int64)
    o = np.argsort(lv, axis=1, kind="stable")
    sv = np.take_along_axis(lv, o, 1)
    ss = np.take_along_axis(ls, o[:, :, None], 1)
    rel = ss - ss[:, :1]
    key = np.concatenate([sv, rel[:, 1:].reshape(-1, 6)], 1)
    uniq, first, counts = np.unique(key, axis=0, return_index=True, return_counts=True)
    assert np.all(counts == 2), "periodic mesh has unmatched facets"
    fac = sv[first]
    fsh = ss[first]
    fmid = (P[fac] + fsh * length).mean(axis=1)
    order = morton_order(np.mod(fmid, length))
    fac, fsh = fac[order], fsh[order]
    spec = MeshSpec(
        vertices=torch.from_numpy(P.astype(np.float32)),
        cells=torch.from_numpy(cells.astype(np.int32)),
        facets=torch.from_numpy(fac.astype(np.int64)),
        bc_facet_mask=torch.zeros(len(fac), dtype=torch.bool),
        bc_tags=[],
        bound_facets=torch.zeros((0, 3), dtype=torch.int64),
        period=np.array([length] * 3),
        cell_shifts=torch.from_numpy(cshift.astype(np.int8)),
        facet_shifts=torch.from_numpy(fsh.astype(np.int8)),
    )
    spec.info = dict(kind="periodic_box", n=n, length=length, seed=seed, jitter=jitter)
    return spec


def periodic_box_cells(n_cells: int, **kw) -> MeshSpec:
    """Periodic box with roughly ``n_cells`` tetrahedra (about 6.5 tetrahedra per grid point)."""
    n = max(4, int(round((n_cells / 6.5) ** (1.0 / 3.0))))
    return periodic_box(n=n, **kw)
