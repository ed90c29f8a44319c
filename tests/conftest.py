import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built librest_b200.so")


def _have_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    """One device context shared by the GPU tests (the library must load: no fallback)."""
    if not _have_gpu():
        pytest.fail("gpu test selected but no CUDA device is visible")
    from rest_b200 import RIJK, build

    build.build()
    c = RIJK(int(os.environ.get("RIJK_TEST_DEVICE", "0")))
    yield c
    c.close()
