import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a path)")


def _has_gpu() -> bool:
    try:
        import symprop_b200 as sp
        return sp.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Session guard for GPU tests: the CUDA library must load and a device
    must be visible; a GPU test never falls back to the CPU."""
    import symprop_b200 as sp
    sp.lib()
    if sp.device_count() == 0:
        pytest.fail("no CUDA device visible to the symprop_b200 library")
    return sp
