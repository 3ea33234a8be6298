import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device and the sm_100a library")


@pytest.fixture(scope="session")
def orc():
    from oracle.oracle import Oracle, build
    build()
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference CPU library (oracle/_ref) not built")
    return Reference()


@pytest.fixture(scope="session")
def lib():
    """The sm_100a library; fails loudly (no fallback) when it is missing."""
    import torch
    import ntt_gpu_b200
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return ntt_gpu_b200.load()
