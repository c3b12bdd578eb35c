"""Canonical forms of per-read results for the tests (the definitions live in oracle/parity.py,
which bench.py's parity check of the benchmarked reads uses as well)."""
from __future__ import annotations

from oracle.parity import canon_from_arrays, canon_from_dump, count_mismatches, diff, f32bits  # noqa: F401


def canon_from_gpu(r) -> tuple[list, list]:
    """The canonical form of mirage_b200.Results."""
    return canon_from_arrays(r.reads, r.cands)
