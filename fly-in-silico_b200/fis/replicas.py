"""Trial replicas across GPUs (one process per GPU).

Trials never exchange data, so the multi-GPU form of the path is replication:
each rank holds the connectome, runs its share of the trials with no
collective on the data path, and the per-trial results are collected on rank
0 at the end (``torch.distributed`` object gather, NCCL or gloo).
"""

from __future__ import annotations


def shard(items, world: int, rank: int):
    """Contiguous share of ``items`` for ``rank``; the first ranks take the remainder."""
    items = list(items)
    q, r = divmod(len(items), world)
    lo = rank * q + min(rank, r)
    hi = lo + q + (1 if rank < r else 0)
    return items[lo:hi], lo


def gather_results(local, world: int, rank: int, dst: int = 0):
    """Gather each rank's ``(offset, results)`` on ``dst``, in trial order."""
    import torch.distributed as dist

    if world == 1:
        return local[1]
    out = [None] * world if rank == dst else None
    dist.gather_object(local, out, dst=dst)
    if rank != dst:
        return None
    merged = []
    for _, res in sorted(out, key=lambda x: x[0]):
        merged.extend(res)
    return merged
