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


def test_results_into_caller_buffers(golden):
    """mg_server_submit_into: the server writes each request's results straight into the
    caller's buffers; they equal the copying form's, alone and mixed with copied requests; a
    candidate buffer too small completes its request with MG_ERR_OOM and the count it needs."""
    g = golden("uneven_small")
    ix = M.Index(g.image)
    rng = np.random.default_rng(9)
    cuts = np.unique(np.concatenate([[0, len(g.reads)], rng.integers(1, len(g.reads), size=30)]))
    parts = split(g.reads, cuts)
    alone = [ix.classify(d, o) for d, o in parts]
    sv = M.Server(ix, max_inflight_reads=1024)
    tickets = [sv.submit_into(d, o) if i % 2 == 0 else sv.submit(d, o) for i, (d, o) in enumerate(parts)]
    assert all(t is not None for t in tickets)
    for a, t in zip(alone, tickets):
        same(a, sv.wait(t))
    big = max(range(len(parts)), key=lambda i: len(alone[i].cands))
    need = len(alone[big].cands)
    assert need > 4
    t = sv.submit_into(*parts[big], cand_cap=need // 2)
    with pytest.raises(M.MirageError) as e:
        sv.wait(t)
    assert e.value.code == -3
    t = sv.submit_into(*parts[big], cand_cap=need)
    same(alone[big], sv.wait(t))
    sv.close()


def test_admission_by_device_budget(golden):
    """A request's device footprint (bases, offsets, results and 8 candidates per read) is booked
    against the server's device budget: one larger than the whole budget is refused for good
    (MG_ERR_LIMIT); while earlier requests hold the budget a new one waits (MG_ERR_BUSY)."""
    g = golden("plain")
    ix = M.Index(g.image)
    d, o = split(g.reads, [0, 2000])[0]
    per = len(d) + 8 * (len(o)) + 2000 * (16 + 8 * 16)
    sv = M.Server(ix, max_inflight_reads=1024, device_budget=int(per * 1.5))
    with pytest.raises(M.MirageError) as e:
        sv.submit(*split(g.reads, [0, 4000])[0])
    assert e.value.code == -4
    t1 = sv.submit(d, o)
    assert t1 is not None
    t2 = None
    for _ in range(2):  # refused while t1 is booked (unless it has completed already)
        t2 = sv.submit(d, o)
        if t2 is None:
            break
        sv.wait(t2)
    same(sv.wait(t1), ix.classify(d, o))
    t3 = sv.submit(d, o)
    assert t3 is not None
    same(sv.wait(t3), ix.classify(d, o))
    sv.close()


def test_bases_read_in_place_from_registered_memory(golden):
    """mg_server_register_host: requests whose bases lie in a range the server page-locked are
    copied to the device from there (only their offsets go through the request ring); their
    results equal the copying path's. The counters of mg_server_get_stats add up: bytes in place
    and through the ring, reads, requests. Memory already page-locked, or registered twice, is
    refused with MG_ERR_INVAL."""
    import torch

    g = golden("uneven_small")
    ix = M.Index(g.image)
    pool = np.array(g.reads.data, dtype=np.uint8, copy=True)  # pageable, owned here
    rng = np.random.default_rng(11)
    cuts = np.unique(np.concatenate([[0, len(g.reads)], rng.integers(1, len(g.reads), size=24)]))
    offs = g.reads.offs
    parts = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        o0, o1 = int(offs[a]), int(offs[b])
        parts.append((pool[o0:o1], (offs[a : b + 1] - offs[a]).astype(np.uint64)))
    alone = [ix.classify(d, o) for d, o in parts]
    sv = M.Server(ix, max_inflight_reads=1024)
    sv.register_host(pool)
    with pytest.raises(M.MirageError) as e:
        sv.register_host(pool)
    assert e.value.code == -8
    pinned = torch.empty(1 << 16, dtype=torch.uint8, pin_memory=True)
    with pytest.raises(M.MirageError) as e:
        sv.register_host(pinned.numpy())
    assert e.value.code == -8
    # even parts in place, odd parts copied (a copy of the slice lies outside the registered range)
    tickets, direct, ring = [], 0, 0
    for i, (d, o) in enumerate(parts):
        src = d if i % 2 == 0 else d.copy()
        t = sv.submit_into(src, o) if i % 3 else sv.submit(src, o)
        assert t is not None
        tickets.append(t)
        if i % 2 == 0:
            direct += len(d)
        else:
            ring += len(d)
    for a, t in zip(alone, tickets):
        same(a, sv.wait(t))
    st = sv.stats()
    assert st["direct_bytes"] == direct and st["ring_bytes"] == ring
    assert st["reads"] == len(g.reads) and st["requests"] == len(parts) and st["steps"] >= 1
    for k in ("submit_copy_s", "launch_s", "device_s", "deliver_s", "idle_s"):
        assert st[k] >= 0.0
    sv.close()
