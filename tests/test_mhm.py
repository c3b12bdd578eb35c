"""The .mhm writer and reader (host code of the product; no GPU needed)."""
import hashlib

import numpy as np
import pytest

import mirage_b200 as M
from conftest import golden_cases


@pytest.mark.parametrize("case", golden_cases())
def test_writer_matches_reference_builder(golden, case):
    """mirage_b200's index build writes the same bytes as the reference's own builder
    (BuildHashmapTable + SaveHashmapTableV3), 32-bit and 64-bit layouts."""
    g = golden(case)
    assert hashlib.sha256(g.image.tobytes()).hexdigest() == g.meta["sha256_mhm"]
    assert len(g.image) == g.meta["mhm_bytes"]


@pytest.mark.parametrize("case", ["plain", "plain64"])
def test_reader_counts(golden, case):
    g = golden(case)
    info = M.inspect_image(g.image, k=31)
    assert info["n_refs"] == g.meta["n_refs"]
    assert info["word"] == g.meta["word"]
    assert info["ref_bases"] == int(g.refs.offs[-1])
    # every indexed position of every reference is one posting (no all-N windows here), except
    # those of the highest hash: the reader gives the last TOC entry BufferSize 0
    # (Hashmap.cpp:552-553) and never decodes its record
    hashes = np.concatenate([hash28_windows(g.refs.seq(r)) for r in range(len(g.refs))])
    last = int(hashes.max())
    assert info["n_postings"] == len(hashes) - int((hashes == last).sum())


def hash28_windows(seq: np.ndarray, h: int = 17) -> np.ndarray:
    """CreateHash24 over every indexed window (positions < len - h) of one reference."""
    n = len(seq) - h
    x = np.full(n, 2166136261, dtype=np.uint64)
    for j in range(h):
        x = ((x * 16777619) & 0xFFFFFFFF) ^ seq[j : j + n].astype(np.uint64)
    return ((x >> 28) ^ x) & 0x0FFFFFFF


def test_reader_rejects_malformed(golden):
    img = golden("plain").image
    with pytest.raises(M.MirageError) as e:
        M.inspect_image(img[:1000], k=31)
    assert e.value.code == -2
    bad = img.copy()
    bad[:6] = np.frombuffer(b"NotMHM", np.uint8)
    with pytest.raises(M.MirageError):
        M.inspect_image(bad, k=31)
    # k below the threshold the index was built with (Hashmap.cpp:457)
    with pytest.raises(M.MirageError):
        M.inspect_image(img, k=21)
    # a truncated posting area (the last record is never decoded, so cut deeper)
    with pytest.raises(M.MirageError):
        M.inspect_image(img[: len(img) * 9 // 10], k=31)


def test_all_n_windows_and_lag():
    """Windows hashing to the all-N hash are skipped without advancing the read pointer
    (Hashmap.cpp:2887-2895): the index build must restate that lag exactly."""
    seq = b"ACGT" * 10 + b"N" * 40 + b"GATTACA" * 12
    bases = np.frombuffer(seq, np.uint8)
    offs = np.array([0, len(seq)], np.uint64)
    img = M.build_image(bases, offs, [b"r0"], k=31)
    info = M.inspect_image(img)
    # simulate the reference loop: i runs over 0..len-18, the window starts at p, p advances
    # only when the window's hash is not the all-N hash
    nnn = int(hash28_windows(np.frombuffer(b"N" * 18, np.uint8))[0])
    kept, p = [], 0
    for i in range(len(seq) - 17):
        h = int(hash28_windows(bases[p : p + 18])[0])
        if h == nnn:
            continue
        kept.append(h)
        p += 1
    assert len(kept) < len(seq) - 17 - 20  # the lag skipped far more than the N run alone
    # postings of the highest hash are never decoded (Hashmap.cpp:552-553)
    assert info["n_postings"] == len(kept) - kept.count(max(kept))


def test_writer_rejects_short_reference():
    bases = np.frombuffer(b"ACGTACGTACGTACGT", np.uint8)
    with pytest.raises(M.MirageError):
        M.build_image(bases, np.array([0, 16], np.uint64), [b"short"], k=31)


def test_word8_roundtrip(golden):
    g = golden("plain")
    img8 = M.build_image(g.refs.data, g.refs.offs, g.refs.headers, k=31, word=8)
    a = M.inspect_image(g.image)
    b = M.inspect_image(img8)
    assert b["word"] == 8 and a["word"] == 4
    for f in ("n_hashes", "n_postings", "n_refs", "ref_bases"):
        assert a[f] == b[f]
