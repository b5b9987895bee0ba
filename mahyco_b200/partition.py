"""Sharing independent cases between GPUs by device memory.

Batched and served cases never exchange data, so N GPUs (one process each)
split them: every case goes to exactly one rank, and the ranks' shares of
device memory (mhc_case_device_bytes, which also tracks the per-cycle
traffic: both scale with the cells and environments) are balanced.  The
only collective is the gathering of per-case results on rank 0 after the
run; nothing crosses between GPUs while they compute.
"""
from __future__ import annotations

import heapq


def partition_by_bytes(sizes: list[int], world: int) -> list[list[int]]:
    """Indices of `sizes` for each of `world` ranks: largest case first, to
    the rank with the fewest bytes so far (ties: the lowest rank); each
    rank's indices in ascending order.  Deterministic, so every rank
    computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + sizes[i], r))
    for part in out:
        part.sort()
    return out


def imbalance(sizes: list[int], parts: list[list[int]]) -> float:
    """Largest rank share over the mean share (1.0 = perfect balance)."""
    loads = [sum(sizes[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def gather_results(local: dict[int, object], world: int, dst: int = 0) -> dict[int, object] | None:
    """Per-case results {case index: value} of every rank, merged on rank
    `dst` (None elsewhere); a rank holding a case index twice, or two ranks
    holding the same index, is an error.  Uses the default process group
    (NCCL or gloo); with one process it returns `local`."""
    import torch.distributed as dist
    if world == 1 or not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    rank = dist.get_rank()
    got = [None] * world if rank == dst else None
    dist.gather_object(local, got, dst=dst)
    if rank != dst:
        return None
    merged: dict[int, object] = {}
    for part in got:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"case {k} was run by two ranks")
            merged[k] = v
    return merged
