import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a B200 (sm_100) and the built libssam_b200.so")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for GPU tests.  A gpu-marked test that finds no device
    fails rather than skips: the CUDA path is the product."""
    import torch
    assert torch.cuda.is_available(), "gpu test run without a CUDA device"
    major, minor = torch.cuda.get_device_capability(0)
    assert major == 10, f"expected an sm_100 device, got sm_{major}{minor}"
    return torch.device("cuda:0")
