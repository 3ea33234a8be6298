"""The butterfly-rate calibration (ntt_b200_butterfly_rate) returns a plausible rate."""
import pytest

import ntt_gpu_b200 as nb

pytestmark = pytest.mark.gpu


def test_butterfly_rate_is_positive_and_repeatable(lib):
    first, second = nb.butterfly_rate(0), nb.butterfly_rate(0)
    assert 1e10 < first < 1e14  # butterflies per second on one GPU
    assert abs(first - second) / first < 0.25
