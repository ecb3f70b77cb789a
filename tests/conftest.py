import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built libliar_gpu.so")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    """One library context on cuda:0 for the whole GPU session."""
    if not _has_gpu():
        pytest.skip("no CUDA device")
    from liar_b200.trace import Context
    ctx = Context(0)
    yield ctx
    ctx.close()
