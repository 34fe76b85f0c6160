import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs with -m gpu")


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for -m gpu tests; fails (never skips) when there is none."""
    import torch
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")


def dev_buffer(nbytes: int):
    import torch
    return torch.zeros(int(nbytes), dtype=torch.uint8, device="cuda:0")
