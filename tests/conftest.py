import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(Path(__file__).resolve().parent) not in sys.path:
    sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


@pytest.fixture(scope="session")
def cuda_lib():
    """The built kinet-b200 library; GPU tests fail (not skip) if it is missing."""
    import crypto_b200

    L = crypto_b200.lib()
    assert crypto_b200.device_available(), "GPU test run without a usable CUDA device"
    return L
