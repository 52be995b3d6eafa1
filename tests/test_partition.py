"""Halo partitioning of one mesh (host logic) and the distributed halo exchange (gloo, 2 ranks)."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import golden_setup


def _parts(case, P):
    from fvm_solver_b200.partition import split_tables
    g, spec, tables, cfg = golden_setup(case)
    return tables.kernel, split_tables(tables.kernel, P)


@pytest.mark.parametrize("case,P", [("c2d", 1), ("c2d", 2), ("c2d", 3), ("b3d", 2), ("b3d", 4)])
def test_partition_invariants(case, P):
    kt, parts = _parts(case, P)
    N = kt.n_cells
    owned = torch.cat([p.cells[:p.n_owned] for p in parts])
    assert torch.equal(torch.sort(owned).values, torch.arange(N))            # every cell owned once
    assert sum(p.tables.n_bc for p in parts) == kt.n_bc                      # every boundary facet once
    assert sum(p.tables.n_char for p in parts) == kt.n_char
    assert all(p.global_n_char == kt.n_char for p in parts)     # same collective plan on every rank
    for p in parts:
        t, n_loc, n_own = p.tables, p.n_local, p.n_owned
        assert t.n_cells == n_loc and n_own > 0
        # facets: both sides local, geometry copied
        assert int(t.fcell.min()) >= 0 and int(t.fcell.max()) < n_loc
        assert torch.equal(t.normals, kt.normals[p.facets])
        assert torch.equal(p.cells[t.fcell.long()], kt.fcell[p.facets].long())
        # every facet of an own cell is local, and maps back to the same global facet
        assert torch.equal(p.facets[t.c2f[:, :n_own].long()], kt.c2f[:, p.cells[:n_own]].long())
        # gradient stencil: weighted columns map back to the same global cell / boundary facet
        cols = t.g_cols[:, :n_own].long()
        w = (t.g_vals[:, :, :n_own] != 0).any(0)
        glob = torch.where(cols < n_loc, p.cells[cols.clamp(max=n_loc - 1)],
                           N + p.bcs[(cols - n_loc).clamp(min=0, max=max(t.n_bc - 1, 0))] if t.n_bc else cols)
        assert torch.equal(glob[w], kt.g_cols[:, p.cells[:n_own]].long()[w])
        # boundary facets: own cells, local facet with the right code side
        if t.n_bc:
            assert int(t.bc_cell.max()) < n_own
            assert torch.equal(p.cells[t.bc_cell.long()], kt.bc_cell[p.bcs].long())
            assert torch.equal(p.facets[t.bc_face.long()], kt.bc_face[p.bcs].long())
        rec = p.records()
        assert rec["cell_rec"].shape[0] == n_loc
        # facet records: geometry and both sides' displacements as in the global records
        grec = kt.records()["face_rec"][p.facets]
        assert torch.equal(rec["face_rec"][:, 2:], grec[:, 2:])
        codes, gcodes = rec["face_rec"][:, :2].view(torch.int32).long(), grec[:, :2].view(torch.int32).long()
        cell_side = codes >= 0
        assert torch.equal(p.cells[codes[cell_side]], gcodes[cell_side])
        assert torch.equal(p.bcs[-1 - codes[~cell_side]], -1 - gcodes[~cell_side])
        # the part's own cell and divergence records equal the global rows
        grec_all = kt.records()
        assert torch.equal(rec["cell_rec"][:n_own, t.kg * t.dim + t.kg:], grec_all["cell_rec"][p.cells[:n_own], t.kg * t.dim + t.kg:])
        # halo rows grouped by owner, matching the owner's send list
        for q, (a, b) in p.recv.items():
            assert torch.equal(parts[q].cells[parts[q].send[p.rank]], p.cells[a:b])
        assert sum(b - a for a, b in p.recv.values()) == n_loc - n_own


def _worker(rank, world, port, case, P_out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from fvm_solver_b200.partition import DistComm
        kt, parts = _parts(case, world)
        part = parts[rank]
        comm = DistComm(part, "cpu")
        buf = torch.full((part.n_local, 4), -1.0)
        buf[:part.n_owned, 0] = part.cells[:part.n_owned].float()
        buf[:part.n_owned, 1] = float(rank)
        comm.exchange([buf])
        ok = torch.equal(buf[:, 0], part.cells.float())
        for q, (a, b) in part.recv.items():
            ok = ok and bool((buf[a:b, 1] == q).all())
        red = torch.tensor([float(rank + 1), float(part.n_owned)], dtype=torch.float64)
        comm.allreduce([red[:1]], "max")
        comm.allreduce([red[1:]], "sum")
        ok = ok and float(red[0]) == world and int(red[1]) == kt.n_cells
        P_out[rank] = int(ok)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,P", [("c2d", 2), ("c2d", 3), ("b3d", 2), ("b3d", 4)])
def test_inner_ranges_need_no_halo(case, P):
    """The overlapped stage runs the inner cells' gradients and the inner facets' fluxes while the
    halo is still being exchanged: their stencils and sides must read no halo row."""
    kt, parts = _parts(case, P)
    for p in parts:
        t, n_loc, n_own = p.tables, p.n_local, p.n_owned
        ni, nf = p.n_inner_cells, p.n_inner_facets
        assert 0 <= ni <= n_own and 0 <= nf <= t.n_facets
        cols = t.g_cols[:, :ni].long()
        w = (t.g_vals[:, :, :ni] != 0).any(0)
        halo_col = (cols >= n_own) & (cols < n_loc)
        assert not bool((halo_col & w).any())
        sides = t.fcell[:nf].long()
        assert not bool(((sides >= n_own) & (sides < n_loc)).any())
        # and the split loses nothing: the other facets each touch a halo cell
        rest = t.fcell[nf:].long()
        assert bool(((rest >= n_own) & (rest < n_loc)).any(1).all())
        # own cells after the inner ones each have a halo cell in their stencil
        cols_o = t.g_cols[:, ni:n_own].long()
        w_o = (t.g_vals[:, :, ni:n_own] != 0).any(0)
        assert bool((((cols_o >= n_own) & (cols_o < n_loc)) & w_o).any(0).all())


@pytest.mark.parametrize("case", ["c2d", "b3d"])
def test_dist_halo_exchange_gloo(case):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Array("i", [0, 0])
    procs = [ctx.Process(target=_worker, args=(r, 2, port, case, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    assert list(out) == [1, 1]
