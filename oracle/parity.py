"""TEST INFRASTRUCTURE ONLY -- canonical forms of per-read results, for bit-exact comparisons
between the reference's dumps (oracle/_ref harness), the CPU restatement and the CUDA path.
Used by tests/ and by bench.py's CPU-baseline leg (the parity check of the benchmarked reads);
the product never imports it.

A strand's canonical form is (HighestScore bits, ((refID, Score bits, percentageMatch bits,
relative-score bits), ...)) over its scored candidates in ascending refID order
(MatrixCPU.cpp:323-370); a read's is (kept strand, merged HighestScore bits, sorted top-group
refIDs) after the strand merge and the top-group pick (Analyser.cpp:592-611, 388-425)."""
from __future__ import annotations

import numpy as np

READ_DTYPE = np.dtype([("highest", "<f4"), ("cand_off", "<u4"), ("n_fwd", "<u2"), ("n_rc", "<u2"),
                       ("strand", "u1"), ("reported", "u1"), ("n_top", "<u2")])
CAND_DTYPE = np.dtype([("ref", "<u4"), ("rel", "<f4"), ("score", "<f4"), ("pct", "<f4")])


def f32bits(x) -> int:
    return int(np.asarray(x, dtype=np.float32).view(np.uint32))


def canon_from_dump(res) -> tuple[list, list]:
    """(strands, reads) from an oracle.Result (reference dump or restatement)."""
    strands = []
    for s in res.strands:
        rel = {ref: rb for rb, ref in s.scores}
        sc = tuple((c[0], c[2], c[3], rel[c[0]]) for c in s.cands if c[3] is not None)
        strands.append((s.highest, sc))
    reads = [(m[1], m[2], tuple(m[3])) for m in res.merged]
    return strands, reads


def canon_from_arrays(reads: np.ndarray, cands: np.ndarray, n: int | None = None) -> tuple[list, list]:
    """The same canonical form from the C ABI's output arrays (mg_read_result, mg_candidate;
    structured arrays or raw bytes) for the first n reads."""
    if reads.dtype != READ_DTYPE:
        reads = np.frombuffer(np.ascontiguousarray(reads).tobytes(), READ_DTYPE)
    if len(cands) and cands.dtype != CAND_DTYPE:
        cands = np.frombuffer(np.ascontiguousarray(cands).tobytes(), CAND_DTYPE)
    n = len(reads) if n is None else n
    cb = cands.view(np.uint32).reshape(-1, 4) if len(cands) else np.zeros((0, 4), np.uint32)
    strands, out = [], []
    for i in range(n):
        rr = reads[i]
        o = int(rr["cand_off"])
        nf, nr = int(rr["n_fwd"]), int(rr["n_rc"])
        his = []
        for a, b in ((o, o + nf), (o + nf, o + nf + nr)):
            his.append(tuple((int(x[0]), int(x[2]), int(x[3]), int(x[1])) for x in cb[a:b]))
        for h in his:
            hi = max((np.uint32(x[3]).view(np.float32) for x in h), default=np.float32(-1))
            strands.append((f32bits(hi), h))
        top = ()
        if rr["reported"]:
            kept = his[int(rr["strand"])]
            top = tuple(sorted(x[0] for x in kept if np.uint32(x[3]).view(np.float32) == rr["highest"]))
        out.append((int(rr["strand"]), f32bits(rr["highest"]), top))
    return strands, out


def diff(a, b, limit: int = 8) -> list[str]:
    """Differences between two canonical forms (empty list = identical)."""
    out = []
    sa, ra = a
    sb, rb = b
    if len(sa) != len(sb):
        return [f"strand count {len(sa)} != {len(sb)}"]
    for i, (x, y) in enumerate(zip(sa, sb)):
        if x != y:
            out.append(f"strand {i} (read {i // 2}): {x} != {y}")
            if len(out) >= limit:
                return out
    for i, (x, y) in enumerate(zip(ra, rb)):
        if x != y:
            out.append(f"read {i}: {x} != {y}")
            if len(out) >= limit:
                return out
    return out


def count_mismatches(a, b) -> dict:
    """Per-field mismatch counts between two canonical forms of the same reads."""
    sa, ra = a
    sb, rb = b
    n = min(len(ra), len(rb))
    strand_bad = sum(1 for x, y in zip(sa, sb) if x != y)
    read_bad = sum(1 for x, y in zip(ra[:n], rb[:n]) if x != y)
    assign_bad = sum(1 for x, y in zip(ra[:n], rb[:n]) if x[2] != y[2])
    return {"reads": n, "strands": min(len(sa), len(sb)), "mismatched_strands": strand_bad,
            "mismatched_reads": read_bad, "mismatched_assignments": assign_bad,
            "mismatches": strand_bad + read_bad + abs(len(ra) - len(rb)) + abs(len(sa) - len(sb))}
