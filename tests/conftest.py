import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def gpu():
    """The CUDA path must be present on a GPU run: a missing library is a
    failure, not a skip (there is no CPU fallback)."""
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    from incrmt_b200 import capi
    capi.lib()  # raises if libincrmt_gpu.so was not built
    return capi


def oracle_available():
    from oracle import refsim
    return refsim.available()
