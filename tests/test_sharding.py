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
