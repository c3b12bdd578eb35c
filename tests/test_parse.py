"""The query-parse restatement against the reference's own parse of the fixtures."""
import glob
import json
import os

import pytest

from parse_util import parse_fasta

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "parse")
CASES = sorted(os.path.basename(p)[:-3] for p in glob.glob(os.path.join(HERE, "*.fa")))


@pytest.mark.parametrize("case", CASES)
def test_restatement_matches_reference_parse(case):
    text = open(os.path.join(HERE, case + ".fa"), "rb").read()
    want = json.load(open(os.path.join(HERE, case + ".json")))
    seqs, hdrs = parse_fasta(text)
    assert [s.decode("latin-1") for s in seqs] == want["sequences"]
    assert [h.decode("latin-1") for h in hdrs] == want["headers"]


def test_restatement_rejects_non_fasta():
    with pytest.raises(ValueError):
        parse_fasta(b"ACGT\n>r1\nGG\n")
    with pytest.raises(ValueError):
        parse_fasta(b">r1\nACGT\n@q\nGG\n")
