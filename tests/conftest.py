import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


def _has_gpu():
    try:
        from gw_fopt_b200 import _lib
        return _lib.lib().bgwx_device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    if not _has_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return True
