"""The index build on the GPU writes the same .mhm bytes as the host builder (which writes the
reference builder's bytes: test_mhm.py)."""
import hashlib

import numpy as np
import pytest

import mirage_b200 as M
from conftest import golden_cases

pytestmark = pytest.mark.gpu


def _same(a: np.ndarray, b: np.ndarray):
    assert len(a) == len(b)
    assert hashlib.sha256(a.tobytes()).hexdigest() == hashlib.sha256(b.tobytes()).hexdigest()


@pytest.mark.parametrize("case", golden_cases())
def test_device_build_equals_reference_builder(golden, case):
    g = golden(case)
    img = M.build_image(g.refs.data, g.refs.offs, g.refs.headers, k=g.meta["k"], word=g.meta["word"], device=0)
    assert hashlib.sha256(img.tobytes()).hexdigest() == g.meta["sha256_mhm"]


def test_device_build_all_n_cutoff_and_taxids():
    """A reference stops being indexed at its first window that hashes like an all-N window
    (Hashmap.cpp:2887-2895); references after it are unaffected; TaxIDs are written as given."""
    rng = np.random.default_rng(3)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    seqs = [acgt[rng.integers(0, 4, 400)].tobytes() + b"N" * 40 + acgt[rng.integers(0, 4, 300)].tobytes(),
            acgt[rng.integers(0, 4, 900)].tobytes(),
            b"N" * 30 + acgt[rng.integers(0, 4, 500)].tobytes(),
            acgt[rng.integers(0, 4, 60)].tobytes()]
    bases = np.frombuffer(b"".join(seqs), np.uint8)
    offs = np.zeros(len(seqs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    names = [b"a", b"bb", b"ccc", b"d"]
    tax = np.array([7, -1, 123456, 42], np.int32)
    for k in (31, 25):
        _same(M.build_image(bases, offs, names, k=k, taxids=tax, device=0),
              M.build_image(bases, offs, names, k=k, taxids=tax))


@pytest.mark.parametrize("k", [15, 19])
def test_device_build_fragmented_rule(k):
    """k < 20 drops the buckets above min(20, the 30th-percentile bucket size)
    (EnableFragmentedDatabase, Hashmap.cpp:1759-1840)."""
    from mirage_b200 import synth

    refs, _, _ = synth.workload("repeats", 0.005, seed=11, n_reads=10)
    _same(M.build_image(refs.data, refs.offs, refs.headers, k=k, device=0),
          M.build_image(refs.data, refs.offs, refs.headers, k=k))


@pytest.mark.parametrize("word", [4, 8])
def test_device_build_large(word):
    from mirage_b200 import synth

    refs, _, _ = synth.workload("uneven_fast", 0.05, seed=2024, n_reads=10)
    _same(M.build_image(refs.data, refs.offs, refs.headers, k=31, word=word, device=0),
          M.build_image(refs.data, refs.offs, refs.headers, k=31, word=word))


MAGIC_LEN = 73  # the .mhm magic text; the bucket TOC starts 24 bytes after it


def _toc_entry(img, i, W=4):
    at = MAGIC_LEN + 24 + 2 * W * i
    return at, int.from_bytes(img[at:at + W].tobytes(), "little"), int.from_bytes(img[at + W:at + 2 * W].tobytes(), "little")


def test_device_open_matches_host_parse(golden):
    for case in ("plain", "plain64"):
        g = golden(case)
        ix = M.Index(g.image)
        host = M.inspect_image(g.image)
        info = ix.info()
        for f in ("n_hashes", "n_postings", "n_refs", "ref_bases", "word"):
            assert info[f] == host[f], f


def test_device_open_rejects_malformed(golden):
    """Malformed images fail to open with MG_ERR_BADFMT, on the device as on the host."""
    img = golden("plain").image
    assert int(img[MAGIC_LEN + 12]) == 4
    _, _, sp0 = _toc_entry(img, 0)
    bad = []
    bad.append(img[: len(img) * 9 // 10])                        # truncated posting area
    b = img.copy(); b[sp0 + 1] = 0; bad.append(b)                # a zero-width refID field
    b = img.copy(); b[sp0 + 3] = 4                               # a 4-byte count of 2^32-1 postings
    wo = int(img[sp0])
    b[sp0 + 4 + 2 * wo:sp0 + 8 + 2 * wo] = 0xFF; bad.append(b)
    at0, _, _ = _toc_entry(img, 0)
    b = img.copy(); b[at0:at0 + 4] = 0xFF; bad.append(b)         # a hash wider than 28 bits
    at1, h1, _ = _toc_entry(img, 1)
    b = img.copy(); b[at0:at0 + 4] = np.frombuffer((h1 + 1).to_bytes(4, "little"), np.uint8); bad.append(b)  # TOC order
    for i, x in enumerate(bad):
        with pytest.raises(M.MirageError) as e:
            M.Index(x)
        assert e.value.code == -2, i
        with pytest.raises(M.MirageError) as e:
            M.inspect_image(x)
        assert e.value.code == -2, i
