import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: large inputs (full benchmark sizes)")


@pytest.fixture(scope="session")
def cuda_device():
    """Fails (does not skip) when no GPU is present: a GPU test that cannot
    reach the CUDA library must not pass silently."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test needs a CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
