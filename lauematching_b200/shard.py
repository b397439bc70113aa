"""Multi-GPU layout of the compare pass: one process per GPU.

The orientation DB shards without communication: rank r holds the contiguous
ID range ``shard_range(n, r, world)`` resident and matches every image of the
batch against it; the per-rank survivor lists are already in ascending ID and
the ranges are ordered by rank, so the global list (the reference's
collection order, LaueMatchingCPU.c:781-788) is the concatenation of the
rank lists in rank order.  That concatenation is the only exchange: a gather
of a few kilobytes per image (over NCCL/NVLink or gloo), no data-path
collective.  The pass-count totals are summed.

Images shard the same way (each rank its own batch against a full DB
replica); that layout needs no exchange at all.
"""
from __future__ import annotations

import numpy as np

__all__ = ["shard_range", "merge_rank_survivors", "gather_survivors"]


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[first, last) of rank's contiguous share of n orientations."""
    base, extra = divmod(n, world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def merge_rank_survivors(per_rank, offsets=None):
    """Concatenate per-rank survivor arrays (ascending local ID) in rank
    order, shifting local IDs by each rank's first global ID."""
    parts = []
    for r, s in enumerate(per_rank):
        s = np.array(s, copy=True)
        if offsets is not None and s.shape[0]:
            s["id"] = s["id"] + np.uint64(offsets[r])
        parts.append(s)
    if not parts:
        return np.zeros(0)
    out = np.concatenate(parts)
    assert np.all(np.diff(out["id"].astype(np.int64)) > 0) if out.shape[0] > 1 else True
    return out


def gather_survivors(local, n_pass: int, first_id: int, group=None):
    """Collective step: every rank contributes (survivors with local IDs,
    pass count, first ID); rank 0 receives the merged global list.

    Returns (merged, total_pass) on every rank (all ranks take the same
    collective steps in the same order)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    items = [None] * world
    dist.all_gather_object(items, (local, int(n_pass), int(first_id)), group=group)
    merged = merge_rank_survivors([it[0] for it in items], [it[2] for it in items])
    return merged, sum(it[1] for it in items)
