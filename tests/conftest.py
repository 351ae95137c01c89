"""Shared pytest configuration: the ``gpu`` marker and repo-root imports."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Skips nothing: a gpu-marked test on a box without a GPU must fail loudly."""
    if not cuda_available():
        pytest.fail("gpu-marked test ran without a CUDA device")
    import rtdl_b200

    rtdl_b200.load_library()
    return True
