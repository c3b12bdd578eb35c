"""Multi-GPU form: index replicas, reads sharded across ranks (one process per GPU).

Reads are independent, so there is no exchange step: each rank classifies a contiguous range of
the reads against its own replica of the index, and results are concatenated in read order
(the reference's node split, Sequences.cpp:1084-1126, does the same across hosts).
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) of n reads for rank (sizes differ by at most one)."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_batch(bases: np.ndarray, offs: np.ndarray, rank: int, world: int):
    """This rank's reads as a CSR batch of their own (offsets rebased to 0)."""
    lo, hi = shard_range(len(offs) - 1, rank, world)
    o0, o1 = int(offs[lo]), int(offs[hi])
    return bases[o0:o1], (offs[lo : hi + 1] - offs[lo]).astype(np.uint64), lo


def concat_results(parts):
    """Concatenate per-rank (reads, cands) arrays in rank order, rebasing cand_off."""
    reads, cands, off = [], [], 0
    for r, c in parts:
        r = r.copy()
        r["cand_off"] += off
        off += len(c)
        reads.append(r)
        cands.append(c)
    return np.concatenate(reads), np.concatenate(cands)
