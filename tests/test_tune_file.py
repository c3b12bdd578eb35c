"""The tuning file's format (written by mirage_b200.tune, read by mg_open); no GPU needed."""
from mirage_b200 import tune as T


def test_tuning_file_keeps_other_classes(tmp_path):
    p = str(tmp_path / "tuning" / "GPU.txt")
    T.write_tuning_file(p, "dense", {"steal_chunk": 8, "first_tier": 1, "not_a_field": 3}, note="a # b")
    T.write_tuning_file(p, "saturated", {"first_tier": 2}, note="sat")
    T.write_tuning_file(p, "dense", {"finish_blocks_per_sm": 4})
    notes = {}
    got = T.read_tuning_file(p, notes)
    assert got == {"dense": {"steal_chunk": 8, "first_tier": 1, "finish_blocks_per_sm": 4},
                   "saturated": {"first_tier": 2}}
    assert notes["dense"] == "a  b" and notes["saturated"] == "sat"
    for line in open(p):
        if not line.startswith("#"):
            cls, *kv = line.split("#")[0].split()
            assert all("=" in x for x in kv)
