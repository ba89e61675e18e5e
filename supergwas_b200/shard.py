"""Weak-scaling shards of one k-mer batch across ranks.

k-mers are independent (the reference already splits them into batch_*
directories, one process each), so ranks take contiguous k-mer ranges and
exchange nothing on the data path.  The only combination step is the one
the reference's merge script performs (HPC/kgwas/merge.sh): concatenate the
output rows in k-mer order and add up the ``.count`` values.
"""
from __future__ import annotations

import numpy as np


def shard_range(m: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, stop) of rank `rank` out of `world`; sizes differ by at most 1."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, rem = divmod(m, world)
    start = rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


def merge(parts):
    """Merge per-shard (start, n_tested, hits) into (n_tested, hits with global k-mer indices)."""
    total = 0
    hits = []
    for start, n_tested, h in sorted(parts, key=lambda p: p[0]):
        total += int(n_tested)
        h = np.array(h, copy=True)
        if h.size:
            h["kmer"] += np.uint64(start)
        hits.append(h)
    out = np.concatenate(hits) if hits else np.zeros(0)
    return total, out
