import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "fesom-c_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def built():
    """Build (if stale) the C-ABI library and the CPU oracle."""
    from fesomc import build
    build.build_library()
    build.build_oracle()
    from fesomc import abi
    return abi.load()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
