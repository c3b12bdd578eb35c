"""Result logs: the library's writer reproduces the reference's own results_Raw.log (written by
the reference's LogMatrixResults through oracle/ref_harness.cpp) byte for byte, from the same
per-read results."""
import gzip
import os

import numpy as np
import pytest

import mirage_b200 as M
from conftest import golden_cases


def results_from_dump(res) -> M.Results:
    """mg_read_result / mg_candidate arrays (the C ABI's layout) from an oracle.Result."""
    n = len(res.merged)
    reads = np.zeros(n, dtype=M.READ_DTYPE)
    cands = []
    for i in range(n):
        per = []
        for s in (0, 1):
            st = res.strands[2 * i + s]
            rel = {ref: rb for rb, ref in st.scores}
            sc = [(c[0], rel[c[0]], c[2], c[3]) for c in st.cands if c[3] is not None]
            per.append(sc)
        m = res.merged[i]
        reads[i]["highest"] = np.uint32(m[2]).view(np.float32)
        reads[i]["cand_off"] = len(cands)
        reads[i]["n_fwd"], reads[i]["n_rc"] = len(per[0]), len(per[1])
        reads[i]["strand"] = m[1]
        reads[i]["reported"] = 1 if m[3] else 0
        reads[i]["n_top"] = len(m[3])
        cands.extend(per[0] + per[1])
    arr = np.zeros(len(cands), dtype=M.CAND_DTYPE)
    for j, (ref, rb, sb, pb) in enumerate(cands):
        arr[j]["ref"] = ref
        arr[j]["rel"] = np.uint32(rb).view(np.float32)
        arr[j]["score"] = np.uint32(sb).view(np.float32)
        arr[j]["pct"] = np.uint32(pb).view(np.float32)
    return M.Results(reads, arr)


@pytest.mark.parametrize("case", golden_cases())
def test_raw_log_matches_reference(golden, case, tmp_path):
    g = golden(case)
    res = results_from_dump(g.dump)
    n = len(g.reads)
    M.write_logs(str(tmp_path), res, np.arange(n), [b">" + h for h in g.reads.headers],
                 [b">" + h for h in g.refs.headers], np.full(len(g.refs), -1, np.int32))
    got = open(os.path.join(tmp_path, "results_Raw.log"), "rb").read()
    exp = gzip.open(os.path.join(g.dir, "raw.log.gz"), "rb").read()
    assert got == exp
    # the threshold files hold subsets of the raw lines
    raw_lines = set(got.splitlines()[1:])
    for kind in ("HighSensitivity", "Balanced", "HighPrecision"):
        lines = open(os.path.join(tmp_path, f"results_{kind}.log"), "rb").read().splitlines()
        assert lines[0] == got.splitlines()[0]
        assert set(lines[1:]) <= raw_lines


def test_tie_group_order_and_taxids(tmp_path):
    """A two-way tie with TaxIDs: the group is ordered by the reference's TaxID comparator."""
    reads = np.zeros(1, dtype=M.READ_DTYPE)
    reads[0] = (0.5, 0, 3, 0, 0, 1, 2)
    cands = np.zeros(3, dtype=M.CAND_DTYPE)
    cands[0] = (0, 0.5, 10.0, 50.0)
    cands[1] = (1, 0.25, 5.0, 50.0)
    cands[2] = (2, 0.5, 10.0, 50.0)
    M.write_logs(str(tmp_path), M.Results(reads, cands), [7], [b">q7"], [b">a", b">b", b">c"],
                 np.array([9606, 562, 9606], np.int32), first_group_only=False)
    lines = open(os.path.join(tmp_path, "results_Raw.log"), "rb").read().splitlines()
    assert lines[1] == b"7;>q7;0.500000;9606;2;>a,>c"
    assert lines[2] == b"7;>q7;0.250000;562;1;>b"
