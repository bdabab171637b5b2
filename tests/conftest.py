"""Test configuration: the ``gpu`` marker and the shared device/oracle helpers."""

from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def gpu_available() -> bool:
    try:
        from ordito_b200 import _lib

        return _lib.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu() -> None:
    """Fails (not skips) a GPU-marked test when no device is visible: the CUDA path is the product."""
    if not gpu_available():
        pytest.fail("no CUDA device visible to libordito_b200 (gpu-marked test)")
