"""Host logic of the served form: the pinned request ring's allocator, checked on the CPU."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "mirage_b200", "csrc")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_ring_regions_never_overlap(tmp_path, seed):
    exe = str(tmp_path / "ring_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "native", "ring_check.cpp"), "-o", exe],
                   check=True)
    out = subprocess.run([exe, str(seed)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
