"""CUDA path against the reference's own results (golden dumps) and the CPU restatement,
through the C ABI. Bit-exact: candidate sets, Score / percentageMatch / relative-score float
bits, strand merge and top group."""
import numpy as np
import pytest

import mirage_b200 as M
from conftest import golden_cases
from parity_util import canon_from_dump, canon_from_gpu, diff

pytestmark = pytest.mark.gpu

_ix = {}


def index_for(g):
    if g.name not in _ix:
        _ix[g.name] = M.Index(g.image, k=g.meta["k"])
    return _ix[g.name]


@pytest.mark.parametrize("case", golden_cases(large=True))
@pytest.mark.parametrize("form", ["batched", "plain"])
def test_gpu_matches_reference(golden, case, form):
    g = golden(case)
    ix = index_for(g)
    r = ix.classify(g.reads.data, g.reads.offs, form=form)
    d = diff(canon_from_gpu(r), canon_from_dump(g.dump))
    assert not d, "\n".join(d)


@pytest.mark.parametrize("case", ["plain", "uneven_small", "long_small"])
def test_forms_agree_bitwise(golden, case):
    g = golden(case)
    ix = index_for(g)
    a = ix.classify(g.reads.data, g.reads.offs, form="batched")
    b = ix.classify(g.reads.data, g.reads.offs, form="plain")
    assert np.array_equal(a.reads.view(np.uint8), b.reads.view(np.uint8))
    assert np.array_equal(a.cands.view(np.uint8), b.cands.view(np.uint8))


def _strand_bytes(raw: bytes, strand: int) -> bytes:
    up = bytes((c - 32) if 96 < c < 128 else c for c in raw)
    if strand == 0:
        return up
    comp = bytes.maketrans(b"ATUGCYRSWKMBDHVN-~", b"TAACGRYSWMKVHDBN-~")
    return up[::-1].translate(comp)


def test_score_candidates_dropin(golden):
    """mg_score_candidates (the CPUGetHighestScore drop-in) on the reference's own candidate
    lists and runs reproduces its Score / percentageMatch / relative scores."""
    g = golden("uneven_small")
    ix = index_for(g)
    dump = g.dump
    q_off, bases, c_off, refs, r_off, runs = [0], [], [0], [], [0], []
    exp = []
    for s in dump.strands:
        i, strand = s.slot // 2, s.slot % 2
        q = _strand_bytes(g.reads.seq(i).tobytes(), strand)
        bases.append(q)
        q_off.append(q_off[-1] + len(q))
        rel = {ref: rb for rb, ref in s.scores}
        for c in s.cands:
            refs.append(c[0])
            for rr in c[4]:
                runs.extend(rr)
            r_off.append(r_off[-1] + len(c[4]))
            exp.append((c[2], c[3], rel.get(c[0])))
        c_off.append(c_off[-1] + len(s.cands))
    score, pct, rel, hi = ix.score_candidates(np.array(q_off), np.frombuffer(b"".join(bases), np.uint8),
                                              np.array(c_off), np.array(refs), np.array(r_off), np.array(runs))
    sb, pb, rb = score.view(np.uint32), pct.view(np.uint32), rel.view(np.uint32)
    bad = 0
    for j, (es, ep, er) in enumerate(exp):
        if es != int(sb[j]):
            bad += 1
        elif ep is not None and (ep != int(pb[j]) or er != int(rb[j])):
            bad += 1
    assert bad == 0
    his = np.array([s.highest for s in dump.strands], dtype=np.uint32)
    assert np.array_equal(hi.view(np.uint32), his)


def test_logf_matches_host_libm_exhaustively(golden):
    """The device logarithm of the relative score equals the host libm logf (which the
    reference calls) at every float in [1, 2^20)."""
    from oracle import oracle as O

    ix = index_for(golden("plain"))
    lo, hi = 0x3F800000, 0x49800000
    step = 1 << 24
    for a in range(lo, hi, step):
        n = min(step, hi - a)
        x = (np.arange(n, dtype=np.uint64) + a).astype(np.uint32).view(np.float32)
        dev = ix.eval_logf(x)
        host = O.logf_bits(a, n)
        mism = np.flatnonzero(dev.view(np.uint32) != host.view(np.uint32))
        assert len(mism) == 0, f"{len(mism)} mismatches from {a:#x}, first at {x[mism[0]]!r}"


@pytest.mark.parametrize("case", ["uneven_small", "repeats_small", "long_small", "uneven_full"])
def test_probe_layouts_agree(golden, case):
    """The dual-strand tiers probe the hash-slot table (count, offset and first 7 postings per
    hash) or the directory and postings arrays; both give the reference's results bit for bit,
    on small indexes (slots forced on) and on the full-scale one (slots forced off)."""
    g = golden(case)
    ix = index_for(g)
    was = bool(ix.info()["probe_slots"])
    try:
        out = {}
        for on in (not was, was):
            ix.set_probe_slots(on)
            assert bool(ix.info()["probe_slots"]) == on
            out[on] = ix.classify(g.reads.data, g.reads.offs)
        assert np.array_equal(out[True].reads.view(np.uint8), out[False].reads.view(np.uint8))
        assert np.array_equal(out[True].cands.view(np.uint8), out[False].cands.view(np.uint8))
        d = diff(canon_from_gpu(out[True]), canon_from_dump(g.dump))
        assert not d, "\n".join(d)
    finally:
        ix.set_probe_slots(was)
