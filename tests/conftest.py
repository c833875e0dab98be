"""Shared fixtures.  `gpu` marks tests that need a CUDA device."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="session")
def ref_available():
    from oracle import refharness
    if not refharness.available():
        pytest.skip("reference oracle library not built (make -C oracle ref)")
    return True
