"""Multi-GPU sharding of independent objects (one process per GPU, ``torch.distributed``).

The benchmarked paths shard as independent objects, so no collective touches the data path:

* ``partition_cases`` -- the batched ensemble's cases are split across ranks balanced by cell
  count (longest-processing-time greedy: largest case to the least-loaded rank); each rank then
  advances its own ``BatchedFVM``.
* ``gather_case_results`` -- the only communication: one all-gather of fixed-size per-case
  result rows at the end, reassembled in global case order on every rank.
* ``run_sharded`` -- the orchestration of one rank: its cases, its batch, the barriers around the
  timed stepping, the max-over-ranks time and the final gather (the batch itself is passed in, so
  the same code drives the CUDA ensemble and the CPU tests).
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


def run_sharded(sizes, steps: int, make_batch, advance, case_rows, row_width: int, device=None,
                group=None) -> dict:
    """One rank's part of a sharded ensemble, with no collective inside the stepping.

    ``sizes`` are the per-case cell counts (every rank passes the same list).  This rank takes the
    cases ``partition_cases`` gives it, builds its batch with ``make_batch(ids)``, then, between two
    barriers, advances it with ``advance(batch, steps)`` -> device milliseconds (timed by the
    caller with events on its stream).  At the end: the time's maximum over ranks and one
    all-gather of ``case_rows(batch)`` ([len(ids), row_width] rows, one per owned case, in ``ids``
    order) into a [n_cases, row_width] float64 tensor in global case order.  A rank without cases
    calls ``make_batch([])`` but neither advances nor reads rows, and contributes 0 ms.
    """
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    ids = partition_cases(sizes, world)[rank]
    batch = make_batch(ids)
    if world > 1:
        dist.barrier(group=group)
    ms = float(advance(batch, steps)) if ids else 0.0
    if world > 1:
        dist.barrier(group=group)
    ms_max = max_over_ranks(ms, device=device, group=group)
    if ids:
        rows = case_rows(batch).to(torch.float64)
    else:
        rows = torch.zeros((0, row_width), dtype=torch.float64, device=device)
    table = gather_case_results(ids, rows, len(sizes), group=group) if world > 1 else rows
    return {"ids": ids, "ms": ms, "ms_max": ms_max, "rows": table,
            "cells_local": int(sum(int(sizes[i]) for i in ids)), "cells_total": int(sum(int(s) for s in sizes))}
