"""Partition of an ensemble's independent members over ranks (one GPU per
rank): longest-processing-time-first bin packing on the members' cell
counts, no collective on the data path, and one gather of the per-member
results at the end.

The members share nothing, so each rank steps its own share with its own
batched launches; the only exchange is the final gather of small per-member
records (torch.distributed.all_gather_object: NCCL on the GPUs, gloo on
host processes).
"""
from __future__ import annotations

import heapq


def lpt(sizes, nparts: int) -> list:
    """Members assigned to nparts parts, largest first, each to the part with
    the least total so far (ties to the lower part).  Returns one ascending
    list of member indices per part; every member is in exactly one part, and
    the largest part total is at most 4/3 of the optimum plus one member."""
    if nparts <= 0:
        raise ValueError("nparts must be positive")
    order = sorted(range(len(sizes)), key=lambda k: (-sizes[k], k))
    heap = [(0, p) for p in range(nparts)]
    parts = [[] for _ in range(nparts)]
    for k in order:
        load, p = heapq.heappop(heap)
        parts[p].append(k)
        heapq.heappush(heap, (load + sizes[k], p))
    return [sorted(q) for q in parts]


def gather_results(local: dict, group=None) -> dict:
    """Merges every rank's {member index: record} into one dict on every
    rank (records must be picklable; keys must not repeat across ranks)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, dict(local), group=group)
    out = {}
    for d in parts:
        for k, v in d.items():
            if k in out:
                raise ValueError(f"member {k} reported by two ranks")
            out[k] = v
    return dict(sorted(out.items()))
