import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) device")


@pytest.fixture(scope="session")
def lib():
    """The product library; GPU tests fail (not skip) when it is missing."""
    from luspice_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def gpu(lib):
    import torch
    assert torch.cuda.is_available(), "GPU test on a machine without a GPU"
    assert lib.lusp_device_count() > 0
    cap = torch.cuda.get_device_capability(0)
    assert cap[0] >= 10, f"needs sm_100, got {cap}"
    return torch.device("cuda:0")
