"""The launch-shape tuner on the GPU: a bounded sweep whose every candidate gives the default
shapes' results bit for bit (tune() checks that), a tuning file that mg_open then applies to a
new index of the same density class, and results unchanged under the tuned shapes."""
import os

import numpy as np
import pytest

import mirage_b200 as M
from mirage_b200 import tune as T

pytestmark = pytest.mark.gpu


def test_tuner_writes_shapes_that_mg_open_applies(golden, tmp_path, monkeypatch):
    g = golden("uneven_small")
    ix = M.Index(g.image)
    _, cls = ix.get_tuning()
    assert cls == "sparse"
    grid = {"first_tier": [2, 1], "steal_chunk": [1, 8], "second_blocks_per_sm": [2], "long_blocks_per_sm": [1]}
    res = T.tune(ix, g.reads, grid, seconds=20.0, reps=2, e2e=True)
    assert res["ms_per_step"] > 0 and len(res["trials"]) >= 2
    path = str(tmp_path / "tuning.txt")
    fields = {**res["fields"], "steal_chunk": 8, "first_tier": 2, "long_blocks_per_sm": 1}
    T.write_tuning_file(path, cls, fields, note="test")
    want = ix.classify(g.reads.data, g.reads.offs)
    monkeypatch.setenv("MG_TUNING_FILE", path)
    ix2 = M.Index(g.image)
    got_fields, cls2 = ix2.get_tuning()
    assert cls2 == cls
    for k, v in fields.items():
        assert got_fields[k] == v, k
    got = ix2.classify(g.reads.data, g.reads.offs)
    assert np.array_equal(got.reads.view(np.uint8), want.reads.view(np.uint8))
    assert np.array_equal(got.cands.view(np.uint8), want.cands.view(np.uint8))
    # a file without an entry for the class leaves the defaults
    T.write_tuning_file(str(tmp_path / "other.txt"), "saturated", {"first_tier": 2})
    monkeypatch.setenv("MG_TUNING_FILE", str(tmp_path / "other.txt"))
    ix3 = M.Index(g.image)
    assert ix3.get_tuning()[0]["first_tier"] == 1
    for x in (ix, ix2, ix3):
        x.close()
