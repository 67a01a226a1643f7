import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """The native library and the CPU oracle are built in-tree once."""
    from slimtracincpp_b200 import build
    build.build()
    build.build_oracle()
    return True


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
