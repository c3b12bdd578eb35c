"""Canonical forms of per-read results, for bit-exact comparisons between the reference's
dumps, the CPU restatement and the CUDA path."""
from __future__ import annotations

import numpy as np


def f32bits(x) -> int:
    return int(np.asarray(x, dtype=np.float32).view(np.uint32))


def canon_from_dump(res) -> tuple[list, list]:
    """(strands, reads) from an oracle.Result (reference dump or restatement).
    strand: (highest_bits, ((ref, score_bits, pct_bits, rel_bits), ...)) over scored candidates
    read:   (kept strand, highest_bits, sorted top refIDs)"""
    strands = []
    for s in res.strands:
        rel = {ref: rb for rb, ref in s.scores}
        sc = tuple((c[0], c[2], c[3], rel[c[0]]) for c in s.cands if c[3] is not None)
        strands.append((s.highest, sc))
    reads = [(m[1], m[2], tuple(m[3])) for m in res.merged]
    return strands, reads


def canon_from_gpu(r) -> tuple[list, list]:
    """The same canonical form from mirage_b200.Results."""
    strands = []
    reads = []
    cb = r.cands.view(np.uint32).reshape(-1, 4) if len(r.cands) else np.zeros((0, 4), np.uint32)
    for i in range(len(r.reads)):
        rr = r.reads[i]
        o = int(rr["cand_off"])
        nf, nr = int(rr["n_fwd"]), int(rr["n_rc"])
        his = []
        for s, (a, b) in enumerate(((o, o + nf), (o + nf, o + nf + nr))):
            rows = cb[a:b]
            sc = tuple((int(x[0]), int(x[2]), int(x[3]), int(x[1])) for x in rows)
            his.append(sc)
        hf = max((np.uint32(x[3]).view(np.float32) for x in his[0]), default=np.float32(-1))
        hr = max((np.uint32(x[3]).view(np.float32) for x in his[1]), default=np.float32(-1))
        strands.append((f32bits(hf), his[0]))
        strands.append((f32bits(hr), his[1]))
        top = tuple(r.top(i))
        reads.append((int(rr["strand"]), f32bits(rr["highest"]), top))
    return strands, reads


def diff(a, b, limit: int = 8) -> list[str]:
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
