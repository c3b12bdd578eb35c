"""mg_score_candidates_noalloc: candidate scoring that allocates no device memory, called through
the C ABI on device buffers and checked bitwise against mg_score_candidates (the entry point
that copies host buffers), on two calls in a row that share the library's fixed working array."""
import ctypes as C

import numpy as np
import pytest

import mirage_b200 as M

pytestmark = pytest.mark.gpu


def _strand_bytes(read: bytes, strand: int) -> bytes:
    up = bytes((c - 32) if 96 < c < 128 else c for c in read)
    if strand == 0:
        return up
    comp = bytes.maketrans(b"ATUGCYRSWKMBDHVN-~", b"TAACGRYSWMKVHDBN-~")
    return up[::-1].translate(comp)


def _inputs(g, strands):
    """Candidate lists and runs of the given dump strands, in mg_score_candidates' layout."""
    q_off, bases, c_off, refs, r_off, runs = [0], [], [0], [], [0], []
    for s in strands:
        q = _strand_bytes(g.reads.seq(s.slot // 2).tobytes(), s.slot % 2)
        bases.append(q)
        q_off.append(q_off[-1] + len(q))
        for c in s.cands:
            refs.append(c[0])
            for rr in c[4]:
                runs.extend(rr)
            r_off.append(r_off[-1] + len(c[4]))
        c_off.append(c_off[-1] + len(s.cands))
    return (np.array(q_off, np.uint64), np.frombuffer(b"".join(bases), np.uint8), np.array(c_off, np.uint64),
            np.array(refs, np.uint32), np.array(r_off, np.uint64), np.array(runs, np.uint32).reshape(-1))


def _noalloc(ix, q_off, bases, c_off, refs, r_off, runs, stream=None, free_delta=None):
    """One call of the no-allocation entry point; device buffers are made here, by the caller.
    stream: a torch.cuda.Stream to pass (None: the index's stream). free_delta: a list that
    receives the change of the device's free memory across the call itself."""
    import torch

    dev = torch.device("cuda:0")

    def up(a):
        a = np.ascontiguousarray(a)
        t = torch.from_numpy(a.view(np.uint8).copy() if a.size else np.zeros(16, np.uint8)).to(dev)
        return t

    ns, nc = len(q_off) - 1, int(c_off[-1])
    d = [up(x) for x in (q_off, bases, c_off, refs, r_off, runs)]
    score = torch.full((max(nc, 1),), 7.0, dtype=torch.float32, device=dev)
    pct = torch.full_like(score, 7.0)
    rel = torch.full_like(score, 7.0)
    hi = torch.full((max(ns, 1),), 7.0, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    L = M.lib()
    fn = L.mg_score_candidates_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint64] + [C.c_void_p] * 11
    free0 = torch.cuda.mem_get_info(dev)[0]
    rc = fn(ix.h, ns, *[t.data_ptr() for t in d], score.data_ptr(), pct.data_ptr(), rel.data_ptr(), hi.data_ptr(),
            stream.cuda_stream if stream is not None else None)
    if free_delta is not None:
        free_delta.append(torch.cuda.mem_get_info(dev)[0] - free0)
    torch.cuda.synchronize()
    out = [t.cpu().numpy()[:n] for t, n in ((score, nc), (pct, nc), (rel, nc), (hi, ns))]
    return rc, out


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_noalloc_matches_scoring_entry_point_twice(golden):
    g = golden("uneven_small")
    ix = M.Index(g.image)
    strands = g.dump.strands
    # first call: the first half of the strands; second call: all of them (the array still holds
    # the first call's contents when the second starts)
    for part in (strands[: len(strands) // 2], strands):
        args = _inputs(g, part)
        want = ix.score_candidates(*args)
        rc, got = _noalloc(ix, *args)
        assert rc == 0, M.lib().mg_last_error()
        assert int(args[2][-1]) > 100
        for w, o in zip(want, got):
            assert np.array_equal(_bits(w), _bits(o))


def test_noalloc_allocates_nothing_and_takes_a_caller_stream(golden):
    """After the first call on the device (which looks up the array's address), further calls
    leave the device's free memory unchanged, on the index's stream and on a stream the caller
    made, and give the same bits as the host-buffer entry point."""
    import torch

    g = golden("uneven_small")
    ix = M.Index(g.image)
    args = _inputs(g, g.dump.strands)
    want = ix.score_candidates(*args)
    rc, _ = _noalloc(ix, *args)  # set-up call
    assert rc == 0, M.lib().mg_last_error()
    side = torch.cuda.Stream()
    for stream in (None, side, side):
        delta = []
        rc, got = _noalloc(ix, *args, stream=stream, free_delta=delta)
        assert rc == 0, M.lib().mg_last_error()
        assert delta == [0]
        for w, o in zip(want, got):
            assert np.array_equal(_bits(w), _bits(o))


def test_both_scoring_entry_points_refuse_a_run_outside_its_query(golden):
    """A run whose Last.Query lies beyond its query (or whose Start.Reference lies beyond its
    reference) is refused with MG_ERR_INVAL by the host-buffer entry point before any copy and
    by the no-allocation one on the device; neither writes outside its buffers."""
    g = golden("uneven_small")
    ix = M.Index(g.image)
    s = next(x for x in g.dump.strands if x.cands and x.cands[0][4])
    q_off, bases, c_off, refs, r_off, runs = _inputs(g, [s])
    L = int(q_off[1])
    for field, value in ((3, L + 40), (0, 0xFFFFFFF0)):
        bad = runs.copy()
        bad[field] = value
        if field == 3:
            bad[1] = min(int(bad[1]), L)  # keep Start.Query <= Last.Query: the run is walked
        with pytest.raises(M.MirageError) as e:
            ix.score_candidates(q_off, bases, c_off, refs, r_off, bad)
        assert e.value.code == -8
        rc, _ = _noalloc(ix, q_off, bases, c_off, refs, r_off, bad)
        assert rc == -8, M.lib().mg_last_error()


def test_noalloc_rejects_queries_beyond_its_limit(golden):
    g = golden("uneven_small")
    ix = M.Index(g.image)
    s = next(x for x in g.dump.strands if x.cands)
    q_off, bases, c_off, refs, r_off, runs = _inputs(g, [s])
    long_q = np.concatenate([bases] * (2049 // len(bases) + 1))[:2049]
    rc, _ = _noalloc(ix, np.array([0, 2049], np.uint64), long_q, c_off, refs, r_off, runs)
    assert rc == -4
    assert b"2048" in M.lib().mg_last_error()
