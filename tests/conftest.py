import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    from tests import golden_cases

    return golden_cases.load()


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library through its C ABI (loads libkronmult_b200.so)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import kronmult_b200

    return kronmult_b200.lib()
