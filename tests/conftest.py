import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs on the GPU box")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the in-tree libraries when a source is newer (no-op on the GPU box,
    where the snapshot already carries them)."""
    from slak_b200 import _paths, build
    missing = [p for p in (_paths.LIB_MESHGEN, _paths.LIB_ORACLE) if not os.path.exists(p)]
    if missing or os.environ.get("SLAK_TEST_REBUILD"):
        build.build_meshgen()
        build.build_oracle()
    yield


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
