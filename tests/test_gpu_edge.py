"""Edge cases of the CUDA path, each checked against the CPU restatement (oracle/)."""
import os

import numpy as np
import pytest

import mirage_b200 as M
from parity_util import canon_from_dump, canon_from_gpu, diff

pytestmark = pytest.mark.gpu

_ix = {}


def plain_index(golden):
    g = golden("plain")
    if "plain" not in _ix:
        from oracle import oracle as O

        _ix["plain"] = (M.Index(g.image), O.Index(g.mhm_path))
    return g, _ix["plain"]


def csr(seqs):
    offs = np.zeros(len(seqs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    data = np.frombuffer(b"".join(seqs), np.uint8) if seqs else np.zeros(0, np.uint8)
    return data, offs


def check_against_oracle(gix, oix, seqs, form="batched"):
    data, offs = csr(seqs)
    r = gix.classify(data, offs, form=form)
    o = oix.classify(data, offs, threads=os.cpu_count() or 1)
    d = diff(canon_from_gpu(r), canon_from_dump(o))
    assert not d, "\n".join(d)
    return r


def test_empty_batch(golden):
    _, (gix, _) = plain_index(golden)
    r = gix.classify(np.zeros(0, np.uint8), np.zeros(1, np.uint64))
    assert len(r.reads) == 0 and len(r.cands) == 0


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_ragged_and_short_reads(golden, form):
    g, (gix, oix) = plain_index(golden)
    ref0 = g.refs.seq(3).tobytes()
    seqs = [ref0[100:100 + n] for n in (1, 17, 30, 31, 32, 45, 46, 61, 62, 76, 150, 151, 299, 320, 321, 1000, 4999)]
    check_against_oracle(gix, oix, seqs, form)


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_lowercase_and_iupac(golden, form):
    g, (gix, oix) = plain_index(golden)
    s = bytearray(g.refs.seq(7).tobytes()[500:800])
    low = bytes(s).lower()
    withn = bytearray(s)
    for p in range(0, 300, 37):
        withn[p] = ord("N")
    iupac = bytearray(s)
    for p, c in zip(range(5, 300, 41), b"RYSWKMBDHV"):
        iupac[p] = c
    check_against_oracle(gix, oix, [low, bytes(withn), bytes(iupac), bytes(s)], form)


def test_invalid_byte_is_rejected(golden):
    g, (gix, _) = plain_index(golden)
    s = g.refs.seq(1).tobytes()[:150]
    data, offs = csr([s, s[:70] + b"X" + s[71:]])
    with pytest.raises(M.MirageError) as e:
        gix.classify(data, offs)
    assert e.value.code == -6


def test_reverse_strand_and_ties(golden):
    """A read copied from a reference's reverse strand is assigned through its reverse
    complement; a read present in two references gives a two-way top group."""
    g, (gix, oix) = plain_index(golden)
    a = g.refs.seq(11).tobytes()[1000:1150]
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    rc = a[::-1].translate(comp)
    r = check_against_oracle(gix, oix, [a, rc])
    assert r.reads[0]["strand"] == 0 and r.reads[1]["strand"] == 1
    assert r.top(0) == r.top(1) == [11]


def test_small_candidate_buffer_reports_need(golden):
    g, (gix, _) = plain_index(golden)
    reads = g.reads.subset(200)
    full = gix.classify(reads.data, reads.offs)
    need = len(full.cands)
    assert need > 10
    with pytest.raises(M.MirageError) as e:
        gix.classify(reads.data, reads.offs, cand_cap=need // 2)
    assert e.value.code == -3


def test_long_reads_go_through_every_tier(golden):
    """Reads beyond the warp tier (block tier) and beyond shared memory (global tier)."""
    g = golden("long_small")
    from oracle import oracle as O

    gix = M.Index(g.image)
    oix = O.Index(g.mhm_path)
    ref = g.refs.seq(int(np.argmax(g.refs.lengths()))).tobytes()
    seqs = [ref[0:20000], ref[5:25005], ref[100:60100]]
    check_against_oracle(gix, oix, seqs)


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_many_candidates_grow_staging_arena(tmp_path, form):
    """Every read matches 24 identical references: 5,000 reads need 120,000 staging entries,
    more than a fresh workspace holds, so the batch runs again with a larger staging arena and
    still equals the oracle."""
    from oracle import oracle as O

    rng = np.random.default_rng(17)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 20000)]
    refs = [core] * 24 + [acgt[rng.integers(0, 4, 20000)] for _ in range(4)]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))])
    path = tmp_path / "dup.mhm"
    image.tofile(path)
    gix = M.Index(image)
    oix = O.Index(str(path))
    starts = rng.integers(0, 20000 - 150, 5000)
    seqs = [core[s:s + 150].tobytes() for s in starts]
    r = check_against_oracle(gix, oix, seqs, form)
    assert (r.reads["n_fwd"] + r.reads["n_rc"]).sum() >= 24 * 5000


def test_warps_with_more_run_records_than_they_walk_together(tmp_path):
    """Every read matches 7 identical references: 56 postings per strand, all kept, and 7 run
    records per read, so a warp's 32 reads hold 224 records, more than the finishing pass walks
    one per lane (128); each read's lane then walks its own. The results equal the oracle."""
    from oracle import oracle as O

    rng = np.random.default_rng(31)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 20000)]
    refs = [core] * 7 + [acgt[rng.integers(0, 4, 20000)] for _ in range(2)]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))])
    path = tmp_path / "seven.mhm"
    image.tofile(path)
    gix = M.Index(image)
    oix = O.Index(str(path))
    starts = rng.integers(0, 20000 - 150, 512)
    seqs = [core[s:s + 150].tobytes() for s in starts]
    r = check_against_oracle(gix, oix, seqs)
    assert (r.reads["n_fwd"] + r.reads["n_rc"] >= 7).all()


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_strands_of_65_to_128_postings(tmp_path, form):
    """Reads whose forward strand gathers 72 postings, 40 of them kept: five copies of the
    reference the reads come from (kept: full diagonal runs) and eight decoy references holding
    every other seed window of each read (never kept: their found indices alternate, so their
    longest run is 1). Such strands exceed the first dual-strand tier's 64 postings and fit the
    second one's 128 (with at most 64 kept); the results equal the oracle."""
    from oracle import oracle as O

    rng = np.random.default_rng(29)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 20000)]
    k, step, hlen, L = 31, 15, 17, 150
    starts = np.arange(100) * 200
    seqs = [core[s:s + L].tobytes() for s in starts]
    ns = (L - k + step - 1) // step
    decoys = []
    for _ in range(8):
        parts = []
        for s in starts:
            for j in range(0, ns, 2):
                parts.append(core[s + j * step:s + j * step + hlen])
                parts.append(acgt[rng.integers(0, 4, 20)])
        decoys.append(np.concatenate(parts))
    refs = [core] * 5 + decoys
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))], k=k)
    path = tmp_path / "decoys.mhm"
    image.tofile(path)
    gix = M.Index(image, k=k)
    oix = O.Index(str(path), k=k)
    hashes = [O.lib().mgo_hash28(q[j * step:j * step + hlen], hlen) for q in seqs for j in range(ns)]
    per_read = gix.bucket_sizes(np.array(hashes, np.uint32)).astype(np.int64).reshape(len(seqs), ns).sum(1)
    assert (per_read > 64).all() and (per_read <= 128).all(), per_read
    r = check_against_oracle(gix, oix, seqs, form)
    assert (r.reads["n_fwd"] >= 5).all()


def _tile(data, offs, times):
    n, nb = len(offs) - 1, int(offs[-1])
    o = np.concatenate([offs[:-1].astype(np.uint64) + np.uint64(k * nb) for k in range(times)] +
                       [np.array([times * nb], np.uint64)])
    return np.tile(data, times), o


def _same(a, b):
    assert np.array_equal(a.reads.view(np.uint8), b.reads.view(np.uint8))
    assert np.array_equal(a.cands.view(np.uint8), b.cands.view(np.uint8))


@pytest.mark.parametrize("copies", [100, 200])
def test_chunked_batch_equals_one_piece(golden, copies):
    """A batch large enough for the chunked form (copies overlapped with classification, candidate
    offsets continued across chunks) equals the plain form and repeats the golden results:
    300,000 reads in 4 equal chunks, 600,000 reads in 8 chunks of weighted sizes."""
    g = golden("uneven_small")
    gix = M.Index(g.image)
    data, offs = _tile(g.reads.data, g.reads.offs, copies)
    big = gix.classify(data, offs)
    _same(big, gix.classify(data, offs, form="plain"))
    one = gix.classify(g.reads.data, g.reads.offs)
    n = len(g.reads.offs) - 1
    assert np.array_equal(big.reads[:n]["highest"].view(np.uint32), one.reads["highest"].view(np.uint32))
    assert np.array_equal(big.reads[-n:]["n_top"], one.reads["n_top"])


def test_chunked_batch_staging_overflow_runs_whole(tmp_path):
    """Every read has 24 candidates: a chunk overflows the staging arena, and the batch is then
    classified in one piece with a larger arena; the result equals the plain form."""
    rng = np.random.default_rng(23)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 20000)]
    refs = [core] * 24 + [acgt[rng.integers(0, 4, 20000)] for _ in range(4)]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    gix = M.Index(M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))]))
    starts = rng.integers(0, 20000 - 150, 270000)
    data = np.concatenate([core[s:s + 150] for s in starts])
    roffs = np.arange(0, 150 * 270001, 150, dtype=np.uint64)
    a = gix.classify(data, roffs)
    assert (a.reads["n_fwd"] + a.reads["n_rc"]).sum() >= 24 * 270000
    _same(a, gix.classify(data, roffs, form="plain"))


def test_long_read_tier_and_its_hand_offs(tmp_path):
    """Reads of 400 bases to 20 kb on four identical references (every posting of a read's
    true region kept four times) and one unrelated one: the long-read tier's smaller size scores
    the reads whose kept postings fit it (up to 1,024 per strand), its larger size those up to
    2,048 (4,000 and 6,000 bases), which hands longer ones to the block tier (12 kb: more kept
    postings) and to the global-memory tier (20 kb: more than 4,096 postings per strand), with
    errors and lowercase bases in some reads; every result equals the oracle's."""
    from oracle import oracle as O

    rng = np.random.default_rng(43)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 40000)]
    refs = [core] * 4 + [acgt[rng.integers(0, 4, 40000)]]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))])
    path = tmp_path / "four.mhm"
    image.tofile(path)
    gix = M.Index(image)
    oix = O.Index(str(path))
    seqs = []
    for n in (400, 1000, 2500, 3800, 4000, 6000, 12000, 20000):
        s0 = int(rng.integers(0, 40000 - n))
        r = core[s0:s0 + n].copy()
        hit = rng.random(n) < 0.02  # substitutions: broken seeds, shorter occurrence runs
        r[hit] = acgt[(np.searchsorted(acgt, r[hit]) + 1) % 4]
        seqs.append(r.tobytes())
        seqs.append(r.tobytes().lower())
    seqs.append(refs[4][1000:9000].tobytes())
    check_against_oracle(gix, oix, seqs)


@pytest.mark.parametrize("first_tier", [1, 2, 3])
def test_strands_of_129_to_256_postings(tmp_path, first_tier):
    """Reads whose forward strand gathers 160 postings, 40 of them kept: five copies of the
    reference the reads come from and thirty decoys holding every other seed window of each read
    (never kept). Such strands pass the 64- and 128-posting dual-strand tiers on to the 256-posting
    one; with first_tier 2 or 3 the reads start at the larger tiers. Every setting equals the
    oracle, and the three settings agree bit for bit."""
    from oracle import oracle as O

    rng = np.random.default_rng(37)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 20000)]
    k, step, hlen, L = 31, 15, 17, 150
    starts = np.arange(100) * 200
    seqs = [core[s:s + L].tobytes() for s in starts]
    ns = (L - k + step - 1) // step
    decoys = []
    for _ in range(30):
        parts = []
        for s in starts:
            for j in range(0, ns, 2):
                parts.append(core[s + j * step:s + j * step + hlen])
                parts.append(acgt[rng.integers(0, 4, 20)])
        decoys.append(np.concatenate(parts))
    refs = [core] * 5 + decoys
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    key = "decoys30"
    if key not in _ix:
        image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))], k=k)
        path = tmp_path / "decoys30.mhm"
        image.tofile(path)
        _ix[key] = (M.Index(image, k=k), O.Index(str(path), k=k))
    gix, oix = _ix[key]
    hashes = [O.lib().mgo_hash28(q[j * step:j * step + hlen], hlen) for q in seqs for j in range(ns)]
    per_read = gix.bucket_sizes(np.array(hashes, np.uint32)).astype(np.int64).reshape(len(seqs), ns).sum(1)
    assert (per_read > 128).all() and (per_read <= 256).all(), per_read
    gix.set_tuning(first_tier=first_tier)
    try:
        r = check_against_oracle(gix, oix, seqs)
    finally:
        gix.set_tuning()
    assert (r.reads["n_fwd"] >= 5).all()


def test_long_reads_with_more_kept_references_than_the_long_tier_holds(tmp_path):
    """Reads of 450-600 bases on 130 identical references: about 3,600 postings per strand, every
    reference kept, more than the long-read tier's table of kept references takes (64), so the
    reads go on to the block tier and, beyond its 128 candidates, to the global tier; the results
    equal the oracle."""
    from oracle import oracle as O

    rng = np.random.default_rng(47)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 5000)]
    refs = [core] * 130 + [acgt[rng.integers(0, 4, 5000)]]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))])
    path = tmp_path / "many.mhm"
    image.tofile(path)
    gix = M.Index(image)
    oix = O.Index(str(path))
    seqs = [core[s:s + n].tobytes() for s, n in zip(rng.integers(0, 4000, 6), (450, 480, 500, 530, 560, 600))]
    r = check_against_oracle(gix, oix, seqs)
    assert (r.reads["n_fwd"] + r.reads["n_rc"] >= 130).all()


def test_packed_upload_equals_plain_upload(golden):
    """mg_classify with pack_bases = 2 (bases packed 2 bits each on host threads, other bytes sent
    as exceptions, unpacked on the device) gives the same bytes as the upload of the bases as
    given: on 165,000 reads in chunks, with lowercase bases, N and IUPAC bytes scattered, and one
    stretch of reads of N only (more exceptions than a chunk's share: that chunk goes up as given);
    a byte without a reverse complement still fails the call."""
    g = golden("uneven_small")
    ix = M.Index(g.image)
    data, offs = _tile(g.reads.data, g.reads.offs, 55)
    data = data.copy()
    rng = np.random.default_rng(53)
    low = rng.random(len(data)) < 0.05
    data[low] = data[low] | 0x20
    for c in b"NRYSWKMBDHV":
        data[rng.integers(0, len(data), 200)] = c
    a, b = int(offs[40000]), int(offs[46000])  # 6,000 reads of N only
    data[a:b] = ord("N")
    want = ix.classify(data, offs)
    ix.set_tuning(pack_bases=2)
    try:
        got = ix.classify(data, offs)
        _same(want, got)
        bad = data.copy()
        bad[int(offs[120000]) + 5] = ord("X")
        with pytest.raises(M.MirageError) as e:
            ix.classify(bad, offs)
        assert e.value.code == -6
    finally:
        ix.set_tuning()


def test_long_reads_past_the_smaller_long_size(tmp_path):
    """The long-read tier runs in two sizes: reads up to 8,192 bases with up to 2,048 postings per
    strand in the smaller, what it hands on (to 20,480 bases and 4,096 postings) in the larger.
    Reads of 8,191, 8,192 and 8,193 bases sit either side of the length bound; 6,000-base reads
    whose even seed windows also lie in ten decoy references (occurrence runs of 1, never kept)
    gather 2,049 to 4,096 postings on the forward strand, so the smaller size hands them to the
    larger. Every result equals the oracle."""
    from oracle import oracle as O

    rng = np.random.default_rng(53)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 30000)]
    k, step, hlen, L = 31, 15, 17, 6000
    starts = [0, 7000, 14000]
    ns = (L - k + step - 1) // step
    decoys = []
    for _ in range(10):
        parts = []
        for s in starts:
            for j in range(0, ns, 2):
                parts.append(core[s + j * step:s + j * step + hlen])
                parts.append(acgt[rng.integers(0, 4, 20)])
        decoys.append(np.concatenate(parts))
    refs = [core] + decoys + [acgt[rng.integers(0, 4, 10000)]]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))], k=k)
    path = tmp_path / "decoys10.mhm"
    image.tofile(path)
    gix, oix = M.Index(image, k=k), O.Index(str(path), k=k)
    heavy = [core[s:s + L].tobytes() for s in starts]
    hashes = [O.lib().mgo_hash28(q[j * step:j * step + hlen], hlen) for q in heavy for j in range(ns)]
    per_read = gix.bucket_sizes(np.array(hashes, np.uint32)).astype(np.int64).reshape(len(heavy), ns).sum(1)
    assert (per_read > 2048).all() and (per_read <= 4096).all(), per_read
    seqs = heavy + [h.lower() for h in heavy]
    seqs += [core[20000:20000 + 8192].tobytes(), core[21000:21000 + 8193].tobytes(), core[20500:20500 + 8191].tobytes()]
    r = check_against_oracle(gix, oix, seqs)
    assert (r.reads["n_fwd"][:3] >= 1).all()


def test_tier_counts_follow_the_reads(golden):
    """mg_last_tier_counts after a one-piece batched call: reads of 1-20 kb pass every dual-strand
    tier and the general warp tier on to the long-read tier (each count at most the batch), and
    a batch of short reads from the plain references leaves the long-read sizes nothing."""
    g = golden("long_small")
    ix = M.Index(g.image)
    long_reads = g.reads.lengths() > 320
    ix.classify(g.reads.data, g.reads.offs)
    c = ix.last_tier_counts()
    n = len(g.reads)
    assert all(0 <= v <= n for v in c.values()), c
    assert c["warp"] >= int(long_reads.sum()) > 0, c
    gp, (pix, _) = plain_index(golden)
    pix.classify(gp.reads.data, gp.reads.offs)
    cp = pix.last_tier_counts()
    assert cp["long_small"] == 0 and cp["long_large"] == 0 and cp["block"] == 0, cp


def test_strands_that_keep_every_reference(tmp_path):
    """A strand whose longest occurrence run is 2 keeps every reference with a posting
    (max(1, hs - 1) = 1): here about 100, more than the long-read tier's table. Two 1,500-base
    reads have their seed windows planted one per reference, seeds 0 and 1 both in reference 0.
    In the first those two lie on different diagonals: no diagonal run of 2 anywhere, so the
    strand has no candidate and the long-read tier finishes the read itself. In the second they
    lie on one diagonal: the read goes on to the block tier, which scores reference 0. Both equal
    the oracle, and the tier counts show the two paths."""
    from oracle import oracle as O

    rng = np.random.default_rng(61)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    k, step, hlen, L = 31, 15, 17, 1500
    ns = (L - k + step - 1) // step
    reads = [acgt[rng.integers(0, 4, L)] for _ in range(2)]
    refs = [acgt[rng.integers(0, 4, 5000)].copy() for _ in range(2 * ns + 2)]
    r0 = refs[0]
    a, b = reads
    r0[100:100 + hlen] = a[0:hlen]                 # seed 0 of the first read ...
    r0[2000:2000 + hlen] = a[step:step + hlen]     # ... and seed 1, on another diagonal
    r0[3000:3000 + step + hlen] = b[0:step + hlen]  # seeds 0 and 1 of the second read, one diagonal
    for j in range(2, ns):
        refs[j][500:500 + hlen] = a[j * step:j * step + hlen]
        refs[ns + j][700:700 + hlen] = b[j * step:j * step + hlen]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))], k=k)
    path = tmp_path / "keepall.mhm"
    image.tofile(path)
    gix, oix = M.Index(image, k=k), O.Index(str(path), k=k)
    r = check_against_oracle(gix, oix, [a.tobytes(), b.tobytes()])
    c = gix.last_tier_counts()
    assert c["warp"] == 2 and c["long_small"] == 1 and c["long_large"] == 1, c
    assert r.reads["n_fwd"][0] == 0 and r.reads["n_fwd"][1] >= 1


def test_long_reads_chunked_by_bases(golden):
    """A host-buffer batch of few but long reads (over 2 x 12.6 Mbp in all, well under 131,072
    reads) is split into chunks by its bases, so that the copy of one chunk overlaps the work on
    the one before; the results equal those of the batch run in one piece, byte for byte."""
    g = golden("long_small")
    ix = M.Index(g.image)
    reps = max(1, int(np.ceil(30e6 / float(g.reads.offs[-1]))))
    lens = g.reads.lengths()
    offs = np.zeros(len(lens) * reps + 1, np.uint64)
    offs[1:] = np.cumsum(np.tile(lens, reps))
    data = np.tile(g.reads.data[: int(g.reads.offs[-1])], reps)
    assert offs[-1] > 2 * 65536 * 192 and len(offs) - 1 < 2 * 65536
    chunked = ix.classify(data, offs)
    ix.set_tuning(chunks=1)
    try:
        whole = ix.classify(data, offs)
    finally:
        ix.set_tuning()
    assert np.array_equal(chunked.reads.view(np.uint8), whole.reads.view(np.uint8))
    assert np.array_equal(chunked.cands.view(np.uint8), whole.cands.view(np.uint8))


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_reads_past_65535_bases(tmp_path, form):
    """Reads of 65,535 bases (the global tier's last length) to 300 kb on four identical 400 kb
    references and a fifth, different one: from 65,536 bases on they go to the oversize tier,
    which the first call turns on, sizes and grows, running the batch again each time. Every
    result equals the oracle's, with substitutions and lowercase bases in some reads, every read
    is assigned, and a second call on the grown workspace repeats the first byte for byte."""
    from oracle import oracle as O

    rng = np.random.default_rng(61)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 400_000)]
    refs = [core] * 4 + [acgt[rng.integers(0, 4, 400_000)]]
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}" for i in range(len(refs))])
    path = tmp_path / "four.mhm"
    image.tofile(path)
    gix = M.Index(image)
    oix = O.Index(str(path))
    seqs = []
    for n in (65_535, 65_536, 70_000, 131_072, 300_000):
        s0 = int(rng.integers(0, 400_000 - n))
        r = core[s0:s0 + n].copy()
        hit = rng.random(n) < 0.02
        r[hit] = acgt[(np.searchsorted(acgt, r[hit]) + 1) % 4]
        seqs.append(r.tobytes())
    seqs.append(seqs[2].lower())
    seqs.append(refs[4][5000:105000].tobytes())
    seqs.append(core[1000:1150].tobytes())
    first = check_against_oracle(gix, oix, seqs, form=form)
    assert first.reads["reported"].all()
    data, roffs = csr(seqs)
    _same(first, gix.classify(data, roffs, form=form))


def test_reads_past_65535_bases_in_chunks(golden):
    """A host-buffer batch of 66-250 kb reads large enough for chunks: a chunk meets reads that the
    oversize tier has no workspace for yet, so the call runs the batch in one piece, which grows
    it (and the odd chunks' workspace); the next call stays in chunks. Both equal the batch in one
    piece, byte for byte, and repeat the reference's results for the first copy."""
    g = golden("ultralong_small")
    ix = M.Index(g.image)
    reps = max(1, int(np.ceil(30e6 / float(g.reads.offs[-1]))))
    data, offs = _tile(g.reads.data, g.reads.offs, reps)
    assert offs[-1] > 2 * 65536 * 192
    first = ix.classify(data, offs)
    second = ix.classify(data, offs)
    ix.set_tuning(chunks=1)
    try:
        whole = ix.classify(data, offs)
    finally:
        ix.set_tuning()
    _same(first, whole)
    _same(second, whole)
    one = ix.classify(g.reads.data, g.reads.offs)
    d = diff(canon_from_gpu(one), canon_from_dump(g.dump))
    assert not d, "\n".join(d)


def test_read_beyond_the_oversize_limit_is_refused(golden):
    """A read of 2,000,001 bases (past the oversize tier's 2,000,000) fails the call with
    MG_ERR_LIMIT; a read of 200 kb on the same index then classifies."""
    g, (gix, _) = plain_index(golden)
    rng = np.random.default_rng(5)
    big = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 2_000_001)].tobytes()
    data, offs = csr([big])
    with pytest.raises(M.MirageError) as e:
        gix.classify(data, offs)
    assert e.value.code == -4
    data, offs = csr([big[:200_000]])
    gix.classify(data, offs)
