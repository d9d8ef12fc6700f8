"""Shared pytest configuration.

Marker `gpu`: the test needs a CUDA device (run with `-m gpu` on a B200).
Everything else runs on CPU.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def core():
    from psacking_b200 import _core
    return _core


@pytest.fixture(scope="session")
def gpu_core(core):
    if core.device_count() < 1:
        pytest.fail("gpu test collected but no CUDA device is visible")
    return core
