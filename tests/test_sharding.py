"""Host-side multi-rank logic on CPU: case partitioning and the result all-gather (gloo, 2 ranks)."""
import os
import socket

import torch
import torch.multiprocessing as tmp

from fvm_solver_b200.sharding import gather_case_results, max_over_ranks, partition_cases


def test_partition_balanced_and_complete():
    from fvm_solver_b200.workloads import ensemble_params
    sizes = [ensemble_params(i)["n_cells"] for i in range(256)]
    for world in (1, 2, 4, 8):
        parts = partition_cases(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
        assert max(loads) / (sum(sizes) / world) < 1.05


def test_partition_more_ranks_than_cases():
    parts = partition_cases([5, 3], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        sizes = [100, 40, 70, 10, 55]
        mine = partition_cases(sizes, world)[rank]
        rows = torch.tensor([[float(i), float(sizes[i]) * 2.0] for i in mine], dtype=torch.float64).reshape(-1, 2)
        out = gather_case_results(mine, rows, len(sizes))
        t = max_over_ranks(1.5 + rank)
        q.put((rank, out.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_gather_two_ranks_gloo():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, out, t in res:
        assert out == [[0.0, 200.0], [1.0, 80.0], [2.0, 140.0], [3.0, 20.0], [4.0, 110.0]]
        assert t == 2.5


class _FakeBatch:
    """Stand-in for a batch of cases: per-case vectors advanced by a fixed affine map."""

    def __init__(self, ids, sizes):
        self.ids = list(ids)
        self.x = [torch.arange(sizes[i], dtype=torch.float64) * (i + 1) for i in ids]

    def step(self, n):
        for _ in range(n):
            self.x = [0.5 * v + 1.0 for v in self.x]


def _rows(b):
    return torch.stack([torch.stack([v.sum(), torch.tensor(float(v.numel()), dtype=torch.float64)]) for v in b.x])


def _sharded_worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    from fvm_solver_b200.sharding import run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        def advance(b, steps):
            b.step(steps)
            return 10.0 * (rank + 1)          # a device time per rank; the max must win
        out = run_sharded(sizes, 3, lambda ids: _FakeBatch(ids, sizes), advance, _rows, row_width=2)
        q.put((rank, out["ids"], out["rows"].tolist(), out["ms_max"], out["cells_total"]))
    finally:
        dist.destroy_process_group()


def _run_world(world, sizes):
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_run_sharded_gloo_matches_serial():
    """The sharded orchestration on 2 gloo ranks (and on 3 ranks with 2 cases: one rank idle) gives
    every rank the same per-case rows as one rank stepping all cases, and the max time."""
    from fvm_solver_b200.sharding import run_sharded
    for world, sizes in ((2, [7, 3, 12, 5, 9]), (3, [4, 6])):
        serial = run_sharded(sizes, 3, lambda ids: _FakeBatch(ids, sizes),
                             lambda b, n: (b.step(n), 1.0)[1], _rows, row_width=2)
        res = _run_world(world, sizes)
        owned = sorted(i for _, ids, _, _, _ in res for i in ids)
        assert owned == list(range(len(sizes)))
        for rank, ids, rows, ms_max, cells in res:
            assert rows == serial["rows"].tolist()
            assert cells == sum(sizes)
            assert ms_max == 10.0 * max(r + 1 for r, i, _, _, _ in res if i)
