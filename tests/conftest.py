import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the library and the oracle in-tree once per session (no-op when fresh)."""
    from cubesphere_b200.build import build_library, build_oracle
    if os.environ.get("CS_SKIP_BUILD") != "1":
        build_library()
        build_oracle()
    yield
