"""Sharding of the batched form across GPUs (one process per GPU).

The matrices of a batch are independent, so the batch shards with no exchange in the
data path: each rank builds a batched plan (``BatchedPlan``) over its own matrices and
runs it on its own GPU.  The partition balances the work by cost n^3 (factor, log det
and inverse are all O(n^3)) with the longest-processing-time-first rule: matrices in
decreasing cost, each to the rank with the least work so far.  The one collective is
the optional gather of the per-matrix results (info words and log dets) to every rank:
a single all-gather of fixed-size padded tensors (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq


def partition_by_cost(sizes, parts: int) -> list[list[int]]:
    """Indices of the matrices of each part (ascending), balanced by sum n^3 with the
    longest-processing-time-first rule.  Deterministic: ties go to the lower part
    index and, among equal costs, to the lower matrix index."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]) ** 3, i))
    heap = [(0, p) for p in range(parts)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        load, p = heapq.heappop(heap)
        out[p].append(i)
        heapq.heappush(heap, (load + int(sizes[i]) ** 3, p))
    return [sorted(ix) for ix in out]


def loads(sizes, partition) -> list[int]:
    """Sum n^3 of every part."""
    return [sum(int(sizes[i]) ** 3 for i in ix) for ix in partition]


def gather_results(local_idx, info, logdet, total: int, device=None):
    """All-gather of per-matrix results: every rank passes the global indices of its
    matrices with their info words and log dets; every rank gets the full arrays
    (info: int64, logdet: float64, length `total`).  One all-gather of padded tensors
    of width max_part (plus a count), so every rank takes the same collective steps."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    dev = torch.device("cpu") if device is None else torch.device(device)
    n_local = torch.tensor([len(local_idx)], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(counts, n_local)
    width = int(max(int(c.item()) for c in counts))
    buf = torch.zeros((3, max(width, 1)), dtype=torch.float64, device=dev)
    k = len(local_idx)
    if k:
        buf[0, :k] = torch.as_tensor(list(local_idx), dtype=torch.float64)
        buf[1, :k] = torch.as_tensor(list(info), dtype=torch.float64)
        buf[2, :k] = torch.as_tensor(list(logdet), dtype=torch.float64)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    info_all = torch.full((total,), -1, dtype=torch.int64)
    logdet_all = torch.full((total,), float("nan"), dtype=torch.float64)
    for c, part in zip(counts, parts):
        m = int(c.item())
        if m == 0:
            continue
        part = part.cpu()
        idx = part[0, :m].to(torch.int64)
        info_all[idx] = part[1, :m].to(torch.int64)
        logdet_all[idx] = part[2, :m]
    return info_all, logdet_all
