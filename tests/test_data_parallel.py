"""Data-parallel corrector training, host side on CPU (gloo, 2 ranks): the flat gradient bucket
averages every parameter's gradient with one all-reduce, and the first rank's weights and
normalisation are broadcast, so ranks that start from different values and see different data end
every iteration with identical weights."""
import os
import socket

import torch
import torch.multiprocessing as tmp

from fvm_solver_b200.corrector import GradBucket, broadcast_from_first


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(100 + rank)              # every rank starts elsewhere
        params = {"W": torch.randn((3, 4), generator=g), "b": torch.randn(5, generator=g)}
        broadcast_from_first(list(params.values()))
        bucket = GradBucket({k: torch.zeros_like(v) for k, v in params.items()})
        bucket.attach(dist.group.WORLD)
        out = {"world": bucket.world, "params0": {k: v.clone() for k, v in params.items()}}
        for it in range(3):
            for k, v in bucket.views.items():                       # this rank's own gradient
                v.copy_(torch.full_like(v, float(rank + 1) * (it + 1)) + torch.arange(v.numel()).view(v.shape))
            bucket.average()
            for k in params:
                params[k] -= 0.1 * bucket.views[k]
        out["grads"] = {k: v.clone() for k, v in bucket.views.items()}
        out["params"] = {k: v.clone() for k, v in params.items()}
        out["aliased"] = bool(bucket.views["b"].data_ptr() == bucket.flat.data_ptr() + 12 * 4)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_grad_bucket_two_ranks_gloo():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = res[0], res[1]
    assert a["world"] == b["world"] == 2
    for k in ("W", "b"):
        assert torch.equal(a["params0"][k], b["params0"][k])       # rank 0's weights everywhere
        assert torch.equal(a["params"][k], b["params"][k])         # and identical after the steps
        n = a["grads"][k].numel()
        want = torch.full((n,), 1.5 * 3) + torch.arange(n)         # mean of ranks' (r + 1) * 3 + index
        assert torch.allclose(a["grads"][k].flatten(), want)
    assert a["aliased"] and b["aliased"]


def test_grad_bucket_single_process_is_identity():
    bucket = GradBucket({"x": torch.ones(4), "y": torch.full((2, 2), 3.0)})
    bucket.attach(None)
    bucket.views["x"].mul_(2)
    bucket.average()
    assert bucket.world == 1
    assert torch.equal(bucket.flat, torch.tensor([2.0, 2, 2, 2, 3, 3, 3, 3]))
