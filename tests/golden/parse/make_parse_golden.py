"""Regenerate the query-parse fixtures from the reference itself (needs the reference build in
oracle/_ref, so it runs in the build container).

Each case is a small FASTA file; the reference's own loader (Sequences::LoadInputFiles through
oracle/_ref/mg_ref_harness --parse-only) parses it, and its forward sequences and headers are
stored as <case>.json beside the input <case>.fa.

Usage: python tests/golden/parse/make_parse_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

import mirage_b200 as M  # noqa: E402
from oracle import oracle as O  # noqa: E402


def random_fasta(seed: int, n: int) -> bytes:
    """Multi-line records with CRLF and LF line ends, lowercase and IUPAC bytes, empty records."""
    rng = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ACGTacgtNRYKMn", np.uint8)
    out = []
    for i in range(n):
        eol = b"\r\n" if rng.random() < 0.3 else b"\n"
        out.append(b">read_%d some description" % i + eol)
        length = 0 if rng.random() < 0.05 else int(rng.integers(1, 400))
        seq = alpha[rng.integers(0, len(alpha), length)].tobytes()
        width = int(rng.integers(20, 120))
        for a in range(0, length, width):
            out.append(seq[a:a + width] + eol)
    return b"".join(out)


CASES = {
    "basic": b">r1 desc\nACGTacgt\nGGTT\n>r2\nTTTTAAAA\n",
    "crlf": b">r1\r\nACGT\r\nGG\r\n>r2\r\nAAAA\r\n",
    "no_final_newline": b">r1\nACGT\n>r2\nGGCC",
    "empty_records": b">r1\n>r2\nACGT\n>r3\nGG\n>r4\n",
    "random": random_fasta(7, 150),
}


def main():
    with tempfile.TemporaryDirectory(prefix="mg_parse_") as tmp:
        rng = np.random.default_rng(1)
        ref = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 2000)]
        img = M.build_image(ref, np.array([0, len(ref)], np.uint64), [b"ref"], k=31)
        mhm = os.path.join(tmp, "ref.mhm")
        img.tofile(mhm)
        for name, text in CASES.items():
            fa = os.path.join(HERE, name + ".fa")
            with open(fa, "wb") as f:
                f.write(text)
            dump = os.path.join(tmp, name + ".dump")
            subprocess.run([O.HARNESS, "--mhm", mhm, "--reads", fa, "--parse-only", "--out", dump, "--logdir",
                            os.path.join(tmp, "log")], check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            seqs, hdrs = [], []
            with open(dump) as f:
                for line in f:
                    p = line.split()
                    if p[0] == "Q":
                        seqs.append(bytes.fromhex(p[2]).decode("latin-1") if len(p) > 2 else "")
                    elif p[0] == "H":
                        hdrs.append(bytes.fromhex(p[1]).rstrip(b"\0").decode("latin-1") if len(p) > 1 else "")
            # the harness appends the reverse complements' headers after the forward ones
            hdrs = hdrs[: len(seqs)]
            with open(os.path.join(HERE, name + ".json"), "w") as f:
                json.dump({"sequences": seqs, "headers": hdrs}, f)
            print(name, len(seqs), "sequences")


if __name__ == "__main__":
    main()
