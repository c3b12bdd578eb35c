import hashlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def golden_cases(large: bool = False):
    """Golden fixture names; large cases (full-scale indexes, GPU tests only) when asked."""
    out = []
    for d in sorted(os.listdir(GOLDEN)):
        meta = os.path.join(GOLDEN, d, "meta.json")
        if os.path.exists(meta):
            with open(meta) as f:
                if large or not json.load(f).get("large"):
                    out.append(d)
    return out


def _fasta_bytes(seqset) -> bytes:
    parts = []
    for i in range(len(seqset)):
        parts.append(b">" + seqset.headers[i] + b"\n" + seqset.seq(i).tobytes() + b"\n")
    return b"".join(parts)


class GoldenCase:
    """A golden fixture: its inputs regenerated from the seed (checked against the recorded
    digests), the .mhm built by mirage_b200's writer (checked against the digest of the index
    the reference's own builder wrote), and the reference's dump."""

    def __init__(self, name: str, tmpdir: str):
        from mirage_b200 import synth

        self.name = name
        self.dir = os.path.join(GOLDEN, name)
        with open(os.path.join(self.dir, "meta.json")) as f:
            self.meta = json.load(f)
        m = self.meta
        self.refs, self.reads, self.truth = synth.workload(m["workload"], m["scale"], seed=m["seed"],
                                                           n_reads=m["n_reads"])
        self.refs_sha = hashlib.sha256(_fasta_bytes(self.refs)).hexdigest()
        self.reads_sha = hashlib.sha256(_fasta_bytes(self.reads)).hexdigest()
        self.tmpdir = tmpdir
        self._image = None
        self._dump = None

    @property
    def image(self) -> np.ndarray:
        if self._image is None:
            import mirage_b200 as M

            # large cases are built by the device build (same bytes as the host writer)
            self._image = M.build_image(self.refs.data, self.refs.offs, self.refs.headers, k=self.meta["k"],
                                        word=self.meta["word"], device=0 if self.meta.get("large") else None)
        return self._image

    @property
    def mhm_path(self) -> str:
        p = os.path.join(self.tmpdir, self.name + ".mhm")
        if not os.path.exists(p):
            self.image.tofile(p)
        return p

    @property
    def dump(self):
        if self._dump is None:
            from oracle import oracle as O

            self._dump = O.parse_dump(os.path.join(self.dir, "ref.dump.gz"))
        return self._dump


_cache = {}


@pytest.fixture(scope="session")
def golden_tmp(tmp_path_factory):
    return str(tmp_path_factory.mktemp("golden"))


@pytest.fixture(scope="session")
def golden(golden_tmp):
    def get(name: str) -> GoldenCase:
        if name not in _cache:
            _cache[name] = GoldenCase(name, golden_tmp)
        return _cache[name]

    return get


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
