"""FASTA parse on the GPU against the reference's own parse (fixtures) and the restatement."""
import glob
import json
import os
import sys

import numpy as np
import pytest

import mirage_b200 as M
from parse_util import parse_fasta

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "parse")
CASES = sorted(os.path.basename(p)[:-3] for p in glob.glob(os.path.join(HERE, "*.fa")))


def _split(bases, offs):
    return [bases[int(offs[i]):int(offs[i + 1])].tobytes() for i in range(len(offs) - 1)]


@pytest.mark.parametrize("case", CASES)
def test_device_parse_matches_reference(case):
    text = open(os.path.join(HERE, case + ".fa"), "rb").read()
    want = json.load(open(os.path.join(HERE, case + ".json")))
    bases, offs, heads = M.parse_fasta(text)
    assert [s.decode("latin-1") for s in _split(bases, offs)] == want["sequences"]
    assert [h.decode("latin-1") for h in heads] == want["headers"]


def test_device_parse_large_random():
    sys.path.insert(0, HERE)
    from make_parse_golden import random_fasta

    text = random_fasta(11, 20000) + b">last\nacgtn"
    for upper in (True, False):
        bases, offs, heads = M.parse_fasta(text, uppercase=upper)
        seqs, hdrs = parse_fasta(text, uppercase=upper)
        assert _split(bases, offs) == seqs
        assert heads == hdrs


def test_device_parse_golden_reads(golden):
    from conftest import _fasta_bytes

    g = golden("uneven_small")
    bases, offs, heads = M.parse_fasta(_fasta_bytes(g.reads))
    assert np.array_equal(offs, g.reads.offs.astype(np.uint64))
    assert np.array_equal(bases, g.reads.data)
    assert heads == [b">" + h for h in g.reads.headers]


def test_device_parse_refusals():
    bases, offs, heads = M.parse_fasta(b"")
    assert len(offs) == 1 and len(heads) == 0
    for bad in (b"ACGT\n>r1\nGG\n", b"@q1\nACGT\n+\nIIII\n", b">r1\nACGT\n@q\nGG\n"):
        with pytest.raises(M.MirageError) as e:
            M.parse_fasta(bad)
        assert e.value.code == -6
