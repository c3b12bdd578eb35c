"""The CPU restatement (oracle/) against the reference's own CPU path on the index shapes the GPU
edge tests use to drive the dual tiers' less common paths: strands of 72 postings of which 40 are
kept (decoy references that hold every other seed window of each read), and reads that match 7
identical references (7 run records per read). The reference runs live through the harness built
from its sources (oracle/_ref); the test is skipped where that build is absent."""
import os

import numpy as np
import pytest

import mirage_b200 as M


def _decoys():
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
    return [core] * 5 + decoys, seqs


def _seven():
    rng = np.random.default_rng(31)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    core = acgt[rng.integers(0, 4, 20000)]
    refs = [core] * 7 + [acgt[rng.integers(0, 4, 20000)] for _ in range(2)]
    starts = rng.integers(0, 20000 - 150, 512)
    return refs, [core[s:s + 150].tobytes() for s in starts]


@pytest.mark.parametrize("shape", ["decoys", "seven"])
def test_oracle_matches_reference_on_stress_shapes(tmp_path, shape):
    from oracle import oracle as O

    if not os.path.exists(O.HARNESS):
        pytest.skip("the reference harness is not built here")
    refs, seqs = _decoys() if shape == "decoys" else _seven()
    offs = np.zeros(len(refs) + 1, np.uint64)
    offs[1:] = np.cumsum([len(r) for r in refs])
    image = M.build_image(np.concatenate(refs), offs, [f"ref{i}".encode() for i in range(len(refs))], k=31)
    mhm = str(tmp_path / "stress.mhm")
    image.tofile(mhm)
    fasta = tmp_path / "reads.fasta"
    fasta.write_bytes(b"".join(b">r%d\n" % i + s + b"\n" for i, s in enumerate(seqs)))
    dump = str(tmp_path / "ref.dump")
    O.run_harness(mhm, str(fasta), out=dump, logdir=str(tmp_path / "logs"))
    ref = O.parse_dump(dump)
    data = np.frombuffer(b"".join(seqs), np.uint8)
    roffs = np.zeros(len(seqs) + 1, np.uint64)
    roffs[1:] = np.cumsum([len(s) for s in seqs])
    res = O.Index(mhm, k=31).classify(data, roffs, threads=os.cpu_count() or 1)
    d = O.compare(res, ref)
    assert not d, "\n".join(d)
