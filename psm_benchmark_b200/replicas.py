"""Multi-GPU plumbing for the replicas-only layout: every rank holds its own
copy of the data graph and matches its own queries; nothing crosses ranks on
the data path. Ranks meet only to take the maximum of their device times
(one all-reduce) and, when a query stream is split, to gather per-query
counts on rank 0."""
from __future__ import annotations


def shard(items, rank: int, world: int):
    """Round-robin share of `items` for `rank` (strong scaling of a stream)."""
    return list(items)[rank::world]


def max_over_ranks(values, dist=None, device: str = "cpu"):
    """Element-wise maximum of a list of floats over all ranks."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def gather_counts(counts, rank: int, world: int, dist=None):
    """Rank 0 receives every rank's list of (query index, count) pairs for a
    round-robin shard and returns the counts in query order; other ranks
    return None."""
    if dist is None:
        return list(counts)
    out = [None] * world
    dist.all_gather_object(out, list(counts))
    if rank != 0:
        return None
    n = sum(len(c) for c in out)
    merged = [None] * n
    for r, cs in enumerate(out):
        for j, c in enumerate(cs):
            merged[r + j * world] = c
    return merged
