import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the native sm_100a kernels")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests run the native library on cuda:0; a missing GPU or
    library is an error, not a skip, when gpu tests are selected."""
    import torch
    assert torch.cuda.is_available(), "gpu test selected but no CUDA device is visible"
    from lightmetrica_b200 import native
    native.lib()
    return torch.device("cuda:0")
