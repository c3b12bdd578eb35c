"""Served form (continuous batching): every request's results are the same alone and in a mix
of concurrent requests, bit for bit, and match the reference's own results."""
import threading

import numpy as np
import pytest

import mirage_b200 as M
from parity_util import canon_from_dump, canon_from_gpu, diff

pytestmark = pytest.mark.gpu


def split(reads, cuts):
    """Sub-batches of a SeqSet at the given read boundaries."""
    out = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        o0, o1 = int(reads.offs[a]), int(reads.offs[b])
        out.append((reads.data[o0:o1], (reads.offs[a : b + 1] - reads.offs[a]).astype(np.uint64)))
    return out


def same(a: M.Results, b: M.Results):
    assert np.array_equal(a.reads.view(np.uint8), b.reads.view(np.uint8))
    assert np.array_equal(a.cands.view(np.uint8), b.cands.view(np.uint8))


def test_requests_alone_and_mixed(golden):
    g = golden("uneven_small")
    ix = M.Index(g.image)
    rng = np.random.default_rng(5)
    cuts = np.unique(np.concatenate([[0, len(g.reads)], rng.integers(1, len(g.reads), size=40)]))
    parts = split(g.reads, cuts)
    alone = [ix.classify(d, o) for d, o in parts]
    # small steps so requests span steps and steps carry several requests
    sv = M.Server(ix, max_inflight_reads=1024)
    tickets = [sv.submit(d, o) for d, o in parts]
    assert all(t is not None for t in tickets)
    mixed = [sv.wait(t) for t in tickets]
    for a, b in zip(alone, mixed):
        same(a, b)
    # concatenated, the mixed results are the reference's own (golden dump)
    reads, cands, off = [], [], 0
    for m in mixed:
        r = m.reads.copy()
        r["cand_off"] += off
        off += len(m.cands)
        reads.append(r)
        cands.append(m.cands)
    whole = M.Results(np.concatenate(reads), np.concatenate(cands))
    d = diff(canon_from_gpu(whole), canon_from_dump(g.dump))
    assert not d, "\n".join(d)
    sv.close()


def test_concurrent_submitters(golden):
    g = golden("plain")
    ix = M.Index(g.image)
    parts = split(g.reads, list(range(0, len(g.reads), 500)) + [len(g.reads)])
    alone = [ix.classify(d, o) for d, o in parts]
    sv = M.Server(ix, max_inflight_reads=2048)
    got = [None] * len(parts)

    def worker(idx):
        for j in idx:
            t = None
            while t is None:
                t = sv.submit(*parts[j])
            got[j] = sv.wait(t)

    th = [threading.Thread(target=worker, args=(list(range(k, len(parts), 4)),)) for k in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for a, b in zip(alone, got):
        same(a, b)
    sv.close()


def test_admission_and_errors(golden):
    g = golden("plain")
    ix = M.Index(g.image)
    sv = M.Server(ix, max_inflight_reads=1024, max_requests=2)
    d, o = split(g.reads, [0, 3000])[0]
    t1 = sv.submit(d, o)
    t2 = sv.submit(d, o)
    assert t1 is not None and t2 is not None
    # a third request is refused while two are tracked
    assert sv.submit(d, o) is None
    sv.wait(t1)
    sv.wait(t2)
    t3 = sv.submit(d, o)
    assert t3 is not None
    same(sv.wait(t3), ix.classify(d, o))
    # unknown ticket
    with pytest.raises(M.MirageError) as e:
        sv.poll(987654)
    assert e.value.code == -8
    # a byte without a reverse complement fails its own request only, also when the request
    # shares a step with another (1024-read steps, 3000-read requests)
    bad = d.copy()
    bad[int(o[2500]) + 3] = ord("X")
    tb = sv.submit(bad, o)
    tg = sv.submit(d, o)
    with pytest.raises(M.MirageError) as e:
        sv.wait(tb)
    assert e.value.code == -6
    same(sv.wait(tg), ix.classify(d, o))
    # empty request completes at once
    t = sv.submit(np.zeros(0, np.uint8), np.zeros(1, np.uint64))
    r = sv.wait(t)
    assert len(r.reads) == 0
    sv.close()
