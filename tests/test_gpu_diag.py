"""Diagnostics on the GPU: the random-gather roofline microbenchmark."""
import pytest

import mirage_b200 as M

pytestmark = pytest.mark.gpu


def test_gather_bandwidth_is_plausible():
    gbs = M.gather_bandwidth(0, 1 << 30)
    # random 32-byte sectors from HBM: well below the ~8 TB/s copy peak, well above a few GB/s
    assert 200.0 < gbs < 10000.0
