"""Test configuration: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs on a CPU-only machine (oracle pins, host logic, ABI surface);
``-m gpu`` needs a CUDA device and exercises libsdpx_b200.so against the oracle.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "sdpx.rs_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    from sdpx_b200 import _lib
    return _lib.load()
