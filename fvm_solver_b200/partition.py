"""One mesh split across ranks: halo-exchange partitioning and the partitioned time stepper.

A mesh too large for one GPU (or stepped by several) is cut into P parts along its Morton cell
order (contiguous, equal-count cell ranges: compact parts with short boundaries).  Part p keeps
its own cells first, then a halo of one cell layer -- every cell that shares a facet with one of
its cells, grouped by owning part -- and every facet and boundary facet touching one of its own
cells.  The part's ``KernelTables`` are the global ones restricted to those and renumbered, so the
kernels run unchanged on it; ``n_owned`` tells them to update only the part's own cells.

One explicit stage on every part is then (the reference's per-step work, ``FVMEquation.forward``
and the stage combination, ``time_fvm/time_solvers/integrators.py:369-393``, split around two
exchanges):

  1. characteristic BC only: each part's sum of the interior sound speed and its count, summed over
     the parts (the reference takes one global mean, ``facet_boundary.py:427``);
  2. halo exchange of the stage input's primitives (rows of ``FVM_ROW`` floats), overlapped with
     the boundary values and the limited gradients of the part's inner cells (stencils inside the
     part), then the limited gradients of the cells next to the halo;
  3. halo exchange of the limited gradients (rows of ``FVM_GROW`` floats) -- facets on the part
     boundary rebuild both sides' facet values from them -- overlapped with the fluxes of the
     inner facets, then the fluxes of the facets on the part boundary;
  4. divergence, stage combination of the own cells (``fvm_stage_phase`` runs each piece);
  5. last stage: the FP64 CFL maximum and conservation sums combined over the parts, then
     ``fvm_stage_finalize`` (every part computes the same dt).

Each part evaluates the facets on its boundary itself (both parts do the same arithmetic on the
same inputs), so the partitioned run gives the single-mesh results: bitwise for meshes without
characteristic boundaries, up to the FP64 summation order of the sound-speed mean otherwise.

Exchanges go through a ``comm`` object: ``LocalComm`` moves rows between parts held by one
process (several parts on one device; the tests' and a single GPU's stand-in for ranks), and
``DistComm`` sends them with ``torch.distributed`` point-to-point operations (NCCL between GPUs,
gloo on CPU), one part per rank.  Halo rows arriving from one part are contiguous, so they are
received in place; sent rows are gathered into one buffer per destination.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import torch

from . import _lib
from .tables import KernelTables, row_sizes


# ---------------------------------------------------------------------------------------------
# Host partitioning
# ---------------------------------------------------------------------------------------------
def partition_cells(n_cells: int, parts: int) -> torch.Tensor:
    """Owner part of every cell: P contiguous ranges of (almost) equal size in cell order."""
    if parts < 1 or parts > n_cells:
        raise ValueError(f"cannot split {n_cells} cells into {parts} parts")
    bounds = torch.linspace(0, n_cells, parts + 1).round().long()
    owner = torch.empty(n_cells, dtype=torch.long)
    for p in range(parts):
        owner[bounds[p]:bounds[p + 1]] = p
    return owner


@dataclass
class MeshPart:
    """One part of a partitioned mesh (host)."""
    rank: int
    parts: int
    n_owned: int
    cells: torch.Tensor            # [n_local] global ids: own cells, then the halo grouped by owner
    facets: torch.Tensor           # [F_local] global facet ids
    bcs: torch.Tensor              # [Fb_local] global boundary-facet indices
    tables: KernelTables           # the part's tables, renumbered
    face_rec: torch.Tensor | None = None       # [F_local][FVM_FACE_REC] facet records (see below)
    global_n_char: int = 0                     # characteristic facets of the whole mesh (same on every part)
    n_inner_cells: int = 0                     # own cells [0, n_inner_cells) have no halo cell in their stencil
    n_inner_facets: int = 0                    # facets [0, n_inner_facets) have no halo cell on either side
    recv: dict = field(default_factory=dict)   # q -> (start, stop): halo rows owned by part q
    send: dict = field(default_factory=dict)   # q -> local ids of own cells part q keeps in its halo

    @property
    def n_local(self) -> int:
        return int(self.cells.numel())

    def records(self) -> dict:
        """Device records of the part: cell and divergence records from its tables, facet records
        from the global ones (a facet record carries both sides' centroid -> facet displacements,
        which for a halo side come from a cell whose own tables the part does not keep)."""
        rec = self.tables.records()
        rec["face_rec"] = self.face_rec
        return rec


def _remap(values: torch.Tensor, table: torch.Tensor, weights: torch.Tensor | None = None) -> torch.Tensor:
    """Global -> local indices.  With ``weights``, slots of weight zero (ELL padding) may point
    anywhere; they are sent to local index 0."""
    out = table[values.long()]
    bad = out < 0
    if weights is not None:
        if bool((bad & (weights != 0)).any()):
            raise RuntimeError("partition: a weighted index points outside the part")
        out = torch.where(bad, torch.zeros_like(out), out)
    elif bool(bad.any()):
        raise RuntimeError("partition: an index points outside the part")
    return out.to(torch.int32)


def split_tables(kt: KernelTables, parts: int, owner: torch.Tensor | None = None) -> list[MeshPart]:
    """Cut ``kt`` (host tables of one mesh) into ``parts`` parts with one-cell halos."""
    N, F, Fb = kt.n_cells, kt.n_facets, kt.n_bc
    owner = partition_cells(N, parts) if owner is None else owner.long()
    fcell = kt.fcell.long()
    g_cols = kt.g_cols.long()                                 # [kg][N]
    face_rec = kt.records()["face_rec"]
    out = []
    for p in range(parts):
        own = torch.nonzero(owner == p).flatten()
        mine = torch.zeros(N, dtype=torch.bool)
        mine[own] = True
        fmask = mine[fcell[:, 0]] | mine[fcell[:, 1]]
        facets = torch.nonzero(fmask).flatten()
        # inner facets (both sides this part's cells or a boundary) first, then the facets on the
        # part boundary; inner cells (stencil within the part) first, then the cells next to the
        # halo -- so the inner work can run while the halo exchange is in flight
        cross = ~(mine[fcell[facets, 0]] & mine[fcell[facets, 1]])
        facets = torch.cat([facets[~cross], facets[cross]])
        n_inner_f = int((~cross).sum())
        sc = g_cols[:, own]
        used = (kt.g_vals[:, :, own] != 0).any(dim=0)
        foreign = used & (sc < N) & ~mine[sc.clamp(max=N - 1)]
        adj = foreign.any(dim=0)
        own = torch.cat([own[~adj], own[adj]])
        n_inner_c = int((~adj).sum())
        # halo: facet neighbours and gradient-stencil cells of own cells that are not own
        near = torch.cat([fcell[facets].flatten(), g_cols[:, own].flatten()])
        near = near[near < N]
        halo_mask = torch.zeros(N, dtype=torch.bool)
        halo_mask[near] = True
        halo_mask &= ~mine
        halo = torch.nonzero(halo_mask).flatten()
        halo = halo[torch.argsort(owner[halo] * N + halo)]          # grouped by owner, ascending id
        cells = torch.cat([own, halo])
        n_own, n_loc = int(own.numel()), int(cells.numel())
        g2l = torch.full((N,), -1, dtype=torch.long)
        g2l[cells] = torch.arange(n_loc)
        bcs = torch.nonzero(mine[kt.bc_cell.long()]).flatten() if Fb else torch.zeros(0, dtype=torch.long)
        b2l = torch.full((max(Fb, 1),), -1, dtype=torch.long)
        b2l[bcs] = torch.arange(bcs.numel())
        f2l = torch.full((F,), -1, dtype=torch.long)
        f2l[facets] = torch.arange(facets.numel())
        chs = kt.bc_char[bcs].long() if Fb else torch.zeros(0, dtype=torch.long)
        chs = torch.sort(chs[chs >= 0]).values
        c2l = torch.full((max(kt.n_char, 1),), -1, dtype=torch.long)
        c2l[chs] = torch.arange(chs.numel())
        # gradient-stencil columns: cells -> local cells, boundary facets -> n_local + local index
        col_table = torch.cat([g2l, torch.where(b2l >= 0, n_loc + b2l, b2l)])

        def cellwise(a: torch.Tensor, fill=0):
            """Per-cell array (cell index last): own cells copied, halo rows filled."""
            res = torch.full((*a.shape[:-1], n_loc), fill, dtype=a.dtype)
            res[..., :n_own] = a[..., own]
            return res

        g_cols_l = torch.zeros((kt.kg, n_loc), dtype=torch.int32)
        g_cols_l[:, :n_own] = _remap(g_cols[:, own], col_table, (kt.g_vals[:, :, own] != 0).any(dim=0))
        c2f_l = torch.zeros((kt.c2f.shape[0], n_loc), dtype=torch.int32)
        c2f_l[:, :n_own] = _remap(kt.c2f[:, own], f2l)
        f_cols_l = torch.zeros((kt.kf, n_loc), dtype=torch.int32)
        f_cols_l[:, :n_own] = _remap(kt.f_cols[:, own], f2l, kt.f_vals[:, own])
        fbc = kt.fbc[facets].long()
        fbc_l = torch.where(fbc >= 0, b2l[fbc.clamp(min=0)], fbc).to(torch.int32)
        bchar = kt.bc_char[bcs].long() if Fb else torch.zeros(0, dtype=torch.long)
        bchar_l = torch.where(bchar >= 0, c2l[bchar.clamp(min=0)], bchar).to(torch.int32)
        t = KernelTables(
            dim=kt.dim, n_comp=kt.n_comp, n_cells=n_loc, n_facets=int(facets.numel()), n_bc=int(bcs.numel()),
            n_char=int(chs.numel()), kg=kt.kg, kf=kt.kf,
            g_vals=cellwise(kt.g_vals), g_cols=g_cols_l, nb_slot=cellwise(kt.nb_slot), disp=cellwise(kt.disp),
            eps=cellwise(kt.eps), c2f=c2f_l, side=cellwise(kt.side), f_vals=cellwise(kt.f_vals), f_cols=f_cols_l,
            inv_h=kt.inv_h[cells].clone(), volumes=kt.volumes[cells].clone(), centroids=kt.centroids[cells].clone(),
            fcell=_remap(fcell[facets], g2l), fbc=fbc_l, normals=kt.normals[facets].clone(),
            fsize=kt.fsize[facets].clone(), xorth=kt.xorth[facets].clone(), inv_d=kt.inv_d[facets].clone(),
            bc_face=_remap(kt.bc_face[bcs], f2l) if Fb else kt.bc_face[:0].clone(),
            bc_side=kt.bc_side[bcs].clone(),
            bc_cell=_remap(kt.bc_cell[bcs], g2l) if Fb else kt.bc_cell[:0].clone(),
            bc_kind=kt.bc_kind[bcs].clone(), bc_b=kt.bc_b[bcs].clone(), bc_l=kt.bc_l[bcs].clone(),
            bc_ga=kt.bc_ga[bcs].clone(), bc_gb=kt.bc_gb[bcs].clone(), bc_char=bchar_l,
            ch_cell=_remap(kt.ch_cell[chs], g2l) if chs.numel() else kt.ch_cell[:0].clone(),
            ch_normal=kt.ch_normal[chs].clone(), ch_rho=kt.ch_rho[chs].clone(), ch_vn=kt.ch_vn[chs].clone(),
            ch_vt=kt.ch_vt[chs].clone(), ch_p=kt.ch_p[chs].clone())
        # facet records: the global rows with the side codes renumbered (cell -> local cell,
        # boundary code -1 - b -> -1 - local b)
        fr = face_rec[facets].clone()
        codes = fr[:, :2].view(torch.int32).long()
        loc = torch.where(codes >= 0, g2l[codes.clamp(min=0)], -1 - b2l[(-1 - codes).clamp(min=0)])
        if bool((loc[codes >= 0] < 0).any()) or bool((loc[codes < 0] >= 0).any()):
            raise RuntimeError("partition: a facet side points outside the part")
        fr[:, :2] = loc.to(torch.int32).view(torch.float32)
        part = MeshPart(rank=p, parts=parts, n_owned=n_own, cells=cells, facets=facets, bcs=bcs, tables=t,
                        face_rec=fr, global_n_char=int(kt.n_char), n_inner_cells=n_inner_c,
                        n_inner_facets=n_inner_f)
        ho = owner[halo]
        for q in range(parts):
            sel = torch.nonzero(ho == q).flatten()
            if sel.numel():
                part.recv[q] = (n_own + int(sel[0]), n_own + int(sel[-1]) + 1)
        out.append(part)
    # send lists: the rows part q receives from p, in q's halo order, as p's local ids
    for q, pq in enumerate(out):
        for p, (a, b) in pq.recv.items():
            glob = pq.cells[a:b]
            gp = torch.full((N,), -1, dtype=torch.long)
            gp[out[p].cells] = torch.arange(out[p].n_local)
            loc = gp[glob]
            if bool((loc < 0).any()) or bool((loc >= out[p].n_owned).any()):
                raise RuntimeError("partition: a halo cell is not owned by its source part")
            out[p].send[q] = loc
    return out


# ---------------------------------------------------------------------------------------------
# Exchanges
# ---------------------------------------------------------------------------------------------
class LocalComm:
    """All parts in this process (one device): halo rows are copied between the parts' buffers."""

    def __init__(self, parts: list[MeshPart], device):
        self.parts = parts
        self.send = [{q: idx.to(device) for q, idx in p.send.items()} for p in parts]

    def exchange(self, bufs: list[torch.Tensor]):
        """bufs[p]: part p's row buffer [n_local][w]; fills every part's halo rows."""
        for p, part in enumerate(self.parts):
            for q, (a, b) in part.recv.items():
                torch.index_select(bufs[q], 0, self.send[q][p], out=bufs[p][a:b])

    def start(self, bufs: list[torch.Tensor]):
        """Begin an exchange whose completion ``finish`` waits for (here: device copies, done at once
        on the current stream)."""
        self.exchange(bufs)

    def finish(self, handle):
        pass

    def allreduce(self, tensors: list[torch.Tensor], op: str):
        """Combine the parts' tensors elementwise (``sum`` / ``max`` / ``min``) into every one."""
        acc = tensors[0].clone()
        for t in tensors[1:]:
            if op == "sum":
                acc += t
            elif op == "max":
                torch.maximum(acc, t, out=acc)
            else:
                torch.minimum(acc, t, out=acc)
        for t in tensors:
            t.copy_(acc)


class DistComm:
    """One part per rank: halo rows travel by ``torch.distributed`` point-to-point operations
    (gathered into one buffer per destination, received in place), reductions by all-reduce."""

    def __init__(self, part: MeshPart, device, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.part = part
        self.group = group
        self.send = {q: idx.to(device) for q, idx in part.send.items()}

    def exchange(self, bufs: list[torch.Tensor]):
        self.finish(self.start(bufs))

    def start(self, bufs: list[torch.Tensor]):
        """Pack the rows each neighbour needs (on the current stream) and post the sends and
        receives; returns a handle for ``finish``.  With NCCL the transfers run on the
        communicator's stream, so kernels launched meanwhile overlap them."""
        dist = self.dist
        buf = bufs[0]
        ops, keep = [], []
        for q, idx in sorted(self.send.items()):
            packed = buf.index_select(0, idx)
            keep.append(packed)
            ops.append(dist.P2POp(dist.isend, packed, q, group=self.group))
        for q, (a, b) in sorted(self.part.recv.items()):
            ops.append(dist.P2POp(dist.irecv, buf[a:b], q, group=self.group))
        return (dist.batch_isend_irecv(ops) if ops else [], keep)

    def finish(self, handle):
        """Make the current stream wait for the transfers (the packed send buffers stay alive
        until then)."""
        reqs, _keep = handle
        for req in reqs:
            req.wait()

    def allreduce(self, tensors: list[torch.Tensor], op: str):
        dist = self.dist
        rop = {"sum": dist.ReduceOp.SUM, "max": dist.ReduceOp.MAX, "min": dist.ReduceOp.MIN}[op]
        dist.all_reduce(tensors[0], op=rop, group=self.group)


# ---------------------------------------------------------------------------------------------
# Partitioned time stepping
# ---------------------------------------------------------------------------------------------
class _PartState:
    """Device tables, scratch and solver buffers of one part."""

    def __init__(self, part: MeshPart, n_k: int, device):
        from .equation import DeviceMesh
        self.part = part
        self.dev = DeviceMesh(part.tables, device, records=part.records())
        self.dev.struct.n_owned = part.n_owned
        # the characteristic-BC scale is the mean over all parts, formed by PartitionedSolver
        self.dev.struct.char_scale_given = 1
        self.work = self.dev.work()
        # copies of the mesh struct for the overlapped stage: inner cells, the other own cells,
        # inner facets, the other facets (fvm_mesh_t cell_lo / n_owned, facet_lo / n_facets)
        mk = lambda: _lib.Mesh.from_buffer_copy(self.dev.struct)
        self.m_inner_cells, self.m_outer_cells = mk(), mk()
        self.m_inner_faces, self.m_outer_faces = mk(), mk()
        if part.n_inner_cells > 0:
            self.m_inner_cells.n_owned = part.n_inner_cells
        else:                                     # no inner cell: the first launch computes boundary values only
            self.m_inner_cells.cell_lo = part.n_owned
        self.m_outer_cells.cell_lo = part.n_inner_cells
        self.m_inner_faces.n_facets = part.n_inner_facets
        self.m_outer_faces.facet_lo = part.n_inner_facets
        N, C = part.n_local, part.tables.n_comp
        R, G = row_sizes(part.tables.dim)
        self.state = torch.zeros((N, C), device=device)
        self.prims = torch.zeros((N, R), device=device)
        self.grads = torch.zeros((N, G), device=device)
        self.k = torch.zeros((max(n_k, 1), N, C), device=device)
        self.dt = torch.zeros(1, device=device)
        self.has_grads = torch.zeros(1, dtype=torch.int32, device=device)
        self.bufs = _lib.SolverBufs(state=_lib.ptr(self.state), prims=_lib.ptr(self.prims),
                                    grads=_lib.ptr(self.grads), k=_lib.ptr(self.k), dt=_lib.ptr(self.dt),
                                    has_grads=_lib.ptr(self.has_grads), cons=None)


class PartitionedSolver:
    """Explicit Runge-Kutta (Butcher tableau, fixed or CFL time step) on a partitioned mesh.

    ``parts``: the parts this process steps (all of them with ``LocalComm``, its own with
    ``DistComm``); ``phys``: an ``fvm_physics_t`` of the gas; ``tab``: an ``fvm_tableau_t`` (not
    adaptive)."""

    def __init__(self, parts: list[MeshPart], comm, phys, tab, device="cuda"):
        if tab.adaptive:
            raise ValueError("adaptive tableaus are not supported on partitioned meshes")
        self.lib = _lib.load()
        self.parts = [_PartState(p, tab.stages, device) for p in parts]
        self.comm = comm
        self.phys = phys
        self.tab = tab
        self.C = parts[0].tables.n_comp
        # decided from the whole mesh, so that every rank takes the same collective steps even when
        # its own part has no characteristic facet
        self.has_char = parts[0].global_n_char > 0

    # -- state in and out ------------------------------------------------------------------------
    def set_state(self, global_state: torch.Tensor):
        """Own rows of every part from a global [N][C] state (global cell order)."""
        for ps in self.parts:
            own = ps.part.cells[:ps.part.n_owned].to(global_state.device)
            ps.state[:ps.part.n_owned].copy_(global_state.index_select(0, own))
            ps.has_grads.zero_()
            _lib.check(self.lib.fvm_state_to_prims(ct.byref(ps.dev.struct), ct.byref(self.phys), _lib.ptr(ps.state),
                                                   _lib.ptr(ps.prims), _lib.stream_ptr()), "fvm_state_to_prims")

    def gather_state(self, out: torch.Tensor):
        """Write every part's own rows into a global [N][C] state."""
        for ps in self.parts:
            own = ps.part.cells[:ps.part.n_owned].to(out.device)
            out.index_copy_(0, own, ps.state[:ps.part.n_owned])

    def set_dt(self, dt: float):
        for ps in self.parts:
            ps.dt.fill_(dt)

    def cfl_dt(self, cfl: float):
        """dt = cfl / max over all parts' cells of inv_h (|u| + c) (min of the parts' dt)."""
        for ps in self.parts:
            _lib.check(self.lib.fvm_cfl_dt(ct.byref(ps.dev.struct), ct.byref(self.phys), _lib.ptr(ps.state),
                                           float(cfl), _lib.ptr(ps.dt), ct.byref(ps.work.struct),
                                           _lib.stream_ptr()), "fvm_cfl_dt")
        self.comm.allreduce([ps.dt for ps in self.parts], "min")

    # -- one step ----------------------------------------------------------------------------------
    def _char_scale(self):
        s = _lib.stream_ptr()
        for ps in self.parts:
            _lib.check(self.lib.fvm_char_partial(ct.byref(ps.dev.struct), ct.byref(self.phys), _lib.ptr(ps.prims),
                                                 ct.byref(ps.work.struct), s), "fvm_char_partial")
        sl = slice(_lib.FVM_RED_DOUBLES + 6, _lib.FVM_RED_DOUBLES + 8)
        self.comm.allreduce([ps.work.red[sl] for ps in self.parts], "sum")
        for ps in self.parts:
            r = ps.work.red
            mean = (r[sl][:1] / r[sl][1:]).float()          # (float)(sum / count), as in k_bc
            r[sl][:1] = (torch.full_like(mean, 10.0) / mean).double()

    def graph_steps(self, n: int):
        """Capture ``n`` steps (kernels, exchanges and reductions) in a CUDA graph; returns a
        callable that replays them.  The state must already be set (``set_state``)."""
        dev = self.parts[0].state.device
        st = torch.cuda.Stream(device=dev)
        st.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(st):
            with torch.cuda.graph(g, stream=st):
                self.step(n)
        torch.cuda.current_stream().wait_stream(st)

        def replay():
            g.replay()

        replay.graph = g
        return replay

    def halo_rows(self) -> int:
        """Rows received per exchange, summed over this process's parts."""
        return sum(ps.part.n_local - ps.part.n_owned for ps in self.parts)

    def _phase(self, ps, mesh, s, phases):
        _lib.check(self.lib.fvm_stage_phase(ct.byref(mesh), ct.byref(self.phys), ct.byref(self.tab), s,
                                            ct.byref(ps.bufs), ct.byref(ps.work.struct), phases, 0,
                                            _lib.stream_ptr()), "fvm_stage_phase")

    def step(self, n: int = 1):
        """``n`` steps.  Each stage overlaps its two halo exchanges with the work that does not
        need the halo: boundary values and the inner cells' gradients run while the primitives are
        exchanged, the inner facets' fluxes while the limited gradients are; the cells and facets
        next to the halo follow each exchange.  (The characteristic-BC mean, a reduction over own
        cells, comes first, so no collective waits behind an exchange.)"""
        S = self.tab.stages
        final_red = self.tab.cfl > 0
        s_ptr = _lib.stream_ptr()
        BC, CELLS, FACES, DIV = _lib.FVM_PHASE_BC, _lib.FVM_PHASE_CELLS, _lib.FVM_PHASE_FACES, _lib.FVM_PHASE_DIV
        for _ in range(n):
            for s in range(S):
                if self.has_char:
                    self._char_scale()
                h = self.comm.start([ps.prims for ps in self.parts])
                for ps in self.parts:
                    self._phase(ps, ps.m_inner_cells, s, BC | CELLS)
                self.comm.finish(h)
                for ps in self.parts:
                    self._phase(ps, ps.m_outer_cells, s, CELLS)
                h = self.comm.start([ps.grads for ps in self.parts])
                for ps in self.parts:
                    self._phase(ps, ps.m_inner_faces, s, FACES)
                self.comm.finish(h)
                for ps in self.parts:
                    self._phase(ps, ps.m_outer_faces, s, FACES)
                    self._phase(ps, ps.dev.struct, s, DIV)
            if final_red:
                self.comm.allreduce([ps.work.red[16:17] for ps in self.parts], "max")
                for ps in self.parts:
                    _lib.check(self.lib.fvm_stage_finalize(ct.byref(ps.dev.struct), ct.byref(self.tab),
                                                           ct.byref(ps.bufs), ct.byref(ps.work.struct), s_ptr),
                               "fvm_stage_finalize")
