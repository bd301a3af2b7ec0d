"""Device diagnostics the benchmark reports beside its rooflines."""
import math

import pytest

pytestmark = pytest.mark.gpu


def test_gather_rate_is_a_plausible_device_rate(lib):
    # random 8-byte loads from an L2-resident array: between 1 and 2,000 G loads/s on any current GPU
    rate = lib.gather_rate(0)
    assert math.isfinite(rate) and 1e9 < rate < 2e12, rate
