import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the B200 kernels)")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
