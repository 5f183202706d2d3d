"""Sharding of one search across ranks (one process per GPU).

The search partitions: subjects are independent, so each rank scans a
contiguous range of subjects holding about 1/world of the residues, with no
collective on the data path.  The per-rank results (counters, HSP CSR) are
merged on rank 0 only when the caller wants the whole answer in one place;
the merge is a concatenation, because HSP records carry subject-relative
offsets and the CSR is per subject.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(offsets: np.ndarray, world: int) -> np.ndarray:
    """Subject boundaries b[0..world]: rank r scans subjects [b[r], b[r+1]),
    cut where the cumulative residue count crosses r/world of the total."""
    offsets = np.asarray(offsets, dtype=np.int64)
    n = len(offsets) - 1
    total = int(offsets[-1])
    cuts = [0]
    for r in range(1, world):
        target = total * r // world
        s = int(np.searchsorted(offsets, target, side="left"))
        cuts.append(min(max(s, cuts[-1]), n))
    cuts.append(n)
    return np.array(cuts, dtype=np.int64)


def local_database(residues: np.ndarray, offsets: np.ndarray, lo: int, hi: int):
    """Residues and rebased offsets of subjects [lo, hi)."""
    off = np.asarray(offsets, dtype=np.int64)
    a, b = int(off[lo]), int(off[hi])
    return np.asarray(residues)[a:b], off[lo:hi + 1] - a


def merge(parts):
    """parts: per-rank (counters [n_r, 3], hsp_off [n_r + 1], hsps [k_r, 6])
    in rank order -> the whole search's (counters, hsp_off, hsps)."""
    counters = np.concatenate([np.asarray(p[0]).reshape(-1, 3) for p in parts]) if parts else np.zeros((0, 3))
    offs, base = [np.zeros(1, dtype=np.int64)], 0
    for p in parts:
        h = np.asarray(p[1], dtype=np.int64)
        offs.append(h[1:] - h[0] + base)
        base += int(h[-1] - h[0])
    hsps = np.concatenate([np.asarray(p[2]).reshape(-1, 6) for p in parts]) if parts else np.zeros((0, 6))
    return counters.astype(np.int32), np.concatenate(offs), hsps.astype(np.int32)


def gather_to_rank0(part, rank: int, world: int):
    """Collects every rank's part on rank 0 (torch.distributed object
    gather; any backend).  Returns the merged result on rank 0, None
    elsewhere."""
    import torch.distributed as dist
    if world == 1:
        return merge([part])
    out = [None] * world if rank == 0 else None
    dist.gather_object(part, out, dst=0)
    return merge(out) if rank == 0 else None
