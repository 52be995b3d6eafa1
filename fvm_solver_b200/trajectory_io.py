"""Trajectory files in the reference's ``Saver`` format (``time_fvm/ds_saving/saving.py:11-88``).

A run directory holds ``mesh_props.npz`` (cells as ``triangles``, ``vertices``, ``centroids``,
facets as ``edges``, boundary-facet midpoints / normals, the boundary mask under the reference's key
``bc_edge_masK`` and the boundary tags ``bc_type_str``) and one ``t_<t:.4g>.npz`` per saved time:
``t``, the per-component mean / standard deviation of the cell primitives (``prim_mean``,
``prim_std``, shape [1, C]) and the z-scored primitives of the cells (``cell_primatives``) and of the
boundary facets (``bc_primatives``, the mean of the facet's two sides) stored as float16.  Files
written here load with the reference's ``load_step`` and vice versa (``load_step`` below).

Boundary-facet values are evaluated for the saved state itself (one residual evaluation on a
scratch gradient buffer); the reference stores those of its last stage evaluation, which differ
from the saved state's by less than one step.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np
import torch

from . import _lib
from .tables import grad_index


def save_mesh_props(eq, save_dir: str, bc_tags=None):
    """``mesh_props.npz`` of an ``FVMEquation`` (``Saver.__init__``, saving.py:20-36)."""
    os.makedirs(save_dir, exist_ok=True)
    m = eq.mesh
    bc = m.bc_facet_mask.cpu().numpy()
    props = {"triangles": m.cells.cpu().numpy(), "vertices": m.vertices.cpu().numpy(),
             "centroids": m.centroids.cpu().numpy(), "edges": m.facets.cpu().numpy(),
             "bc_midpoints": m.midpoints[bc].cpu().numpy(), "bc_normals": m.normals[bc].cpu().numpy(),
             "bc_edge_masK": bc, "bc_type_str": np.array([] if bc_tags is None else list(bc_tags))}
    np.savez_compressed(os.path.join(save_dir, "mesh_props.npz"), **props)


def boundary_face_values(eq, prims: torch.Tensor) -> torch.Tensor:
    """Mean of the two sides' values of every boundary facet [Fb, C] for the primitives ``prims``."""
    kt = eq.tables.kernel
    Fb, C, dim = kt.n_bc, eq.n_comp, eq.mesh.dim
    if Fb == 0:
        return torch.zeros((0, C), device=prims.device)
    grads = torch.zeros_like(eq.grads)
    flag = torch.zeros(1, dtype=torch.int32, device=prims.device)
    out = torch.empty_like(prims)
    _lib.check(eq.lib.fvm_residual(ct.byref(eq.dev.struct), ct.byref(eq.phys), _lib.ptr(prims), _lib.ptr(grads),
                                   _lib.ptr(flag), _lib.ptr(out), ct.byref(eq.work.struct), _lib.stream_ptr()),
               "fvm_residual")
    bcv = eq.work.bc_vals[:Fb, :C]
    dev = prims.device
    cells = kt.bc_cell.long().to(dev)
    faces = kt.bc_face.long().to(dev)
    # the facet's centroid -> facet displacement seen from its cell
    c2f = kt.c2f.long().to(dev)                        # [K][N]
    disp = kt.disp.to(dev)                             # [K][dim][N]
    j = (c2f[:, cells] == faces.unsqueeze(0)).long().argmax(dim=0)
    r = disp[j, :, cells]                              # [Fb][dim]
    gidx = torch.tensor([[grad_index(dim, d, c) for c in range(C)] for d in range(dim)], device=dev)
    g = grads[cells][:, gidx]                          # [Fb][dim][C]
    inner = prims[cells] + (g * r.unsqueeze(-1)).sum(dim=1)
    return (inner + bcv) / 2


class TrajectorySaver:
    """Writes ``t_<t>.npz`` snapshots of an ``FVMEquation``'s state (``Saver.save``, saving.py:46-72)."""

    def __init__(self, eq, save_dir: str, bc_tags=None):
        self.eq = eq
        self.save_dir = save_dir
        save_mesh_props(eq, save_dir, bc_tags)

    def save(self, t: float, state: torch.Tensor | None = None) -> str:
        eq = self.eq
        state = eq.cells.state if state is None else state
        prims = eq.phy_setup.state_to_primative(state)[0].contiguous()
        bc_vals = boundary_face_values(eq, prims)
        return write_snapshot(self.save_dir, t, prims, bc_vals)


def write_snapshot(save_dir: str, t: float, prims: torch.Tensor, bc_vals: torch.Tensor) -> str:
    """One ``t_<t:.4g>.npz`` file: z-scored fp16 cell and boundary-facet primitives."""
    mean = prims.mean(dim=0, keepdim=True)
    std = prims.std(dim=0, keepdim=True)
    safe = std.clamp(min=1e-8)
    values = {"t": float(t), "prim_mean": mean.cpu().numpy(), "prim_std": std.cpu().numpy(),
              "cell_primatives": ((prims - mean) / safe).cpu().half().numpy(),
              "bc_primatives": ((bc_vals - mean) / safe).cpu().half().numpy()}
    path = os.path.join(save_dir, f"t_{float(t):.4g}.npz")
    np.savez_compressed(path, **values)
    return path


def load_step(file_path: str):
    """(t, cell primitives [N, C], boundary-facet primitives [Fb, C]) of one snapshot file."""
    data = np.load(file_path)
    mean, std = data["prim_mean"], data["prim_std"]
    cell = data["cell_primatives"].astype(np.float32) * std + mean
    bc = data["bc_primatives"].astype(np.float32) * std + mean
    return data["t"], torch.from_numpy(cell).float(), torch.from_numpy(bc).float()
