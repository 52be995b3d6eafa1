"""Multi-GPU sharding of independent objects (one process per GPU, ``torch.distributed``).

The benchmarked paths shard as independent objects, so no collective touches the data path:

* ``partition_cases`` -- the batched ensemble's cases are split across ranks balanced by cell
  count (longest-processing-time greedy: largest case to the least-loaded rank); each rank then
  advances its own ``BatchedFVM``.
* ``gather_case_results`` -- the only communication: one all-gather of fixed-size per-case
  result rows at the end, reassembled in global case order on every rank.
* the 3D box benchmark runs one independent box per rank (weak scaling).

Time is always taken on the device and reduced with MAX over ranks.
"""
from __future__ import annotations

import heapq

import torch


def partition_cases(sizes, world: int) -> list:
    """Case indices per rank, balancing the summed ``sizes``; each list is sorted."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(x) for x in out]


def gather_case_results(local_ids, local_rows: torch.Tensor, n_cases: int, group=None) -> torch.Tensor:
    """All-gather per-case result rows [n_local, W] into a [n_cases, W] tensor in case order.

    Works with any backend (``gloo`` on CPU tensors, ``nccl`` on CUDA tensors).  Ranks may own
    different numbers of cases; rows are padded to the largest share for the collective.
    """
    import torch.distributed as dist
    world = dist.get_world_size(group)
    W = local_rows.shape[1]
    dev = local_rows.device
    n_local = torch.tensor([len(local_ids)], device=dev, dtype=torch.int64)
    counts = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(counts, n_local, group=group)
    mx = int(max(int(c.item()) for c in counts))
    ids = torch.full((mx,), -1, device=dev, dtype=torch.int64)
    ids[:len(local_ids)] = torch.as_tensor(list(local_ids), device=dev, dtype=torch.int64)
    rows = torch.zeros((mx, W), device=dev, dtype=local_rows.dtype)
    rows[:len(local_ids)] = local_rows
    all_ids = [torch.empty_like(ids) for _ in range(world)]
    all_rows = [torch.empty_like(rows) for _ in range(world)]
    dist.all_gather(all_ids, ids, group=group)
    dist.all_gather(all_rows, rows, group=group)
    out = torch.full((n_cases, W), float("nan"), device=dev, dtype=local_rows.dtype)
    for i_, r_ in zip(all_ids, all_rows):
        keep = i_ >= 0
        out[i_[keep]] = r_[keep]
    return out


def max_over_ranks(x: float, device=None, group=None) -> float:
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
