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


def reference_src():
    """The reference's source tree, for checks that read its shipped assets
    in place: $SLIM_REFERENCE_SRC, else the tree oracle/build_ref.sh read
    (recorded in oracle/_ref/reference_src.txt); None when neither exists."""
    cand = os.environ.get("SLIM_REFERENCE_SRC")
    rec = ROOT / "oracle" / "_ref" / "reference_src.txt"
    if not cand and rec.exists():
        cand = rec.read_text().strip()
    return Path(cand) if cand and Path(cand).is_dir() else None
