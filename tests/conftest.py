import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")


def _ensure_built():
    """Build the native libraries if they are missing or stale (a no-op on a prebuilt tree)."""
    from simpler_b200 import build
    build.build_library()
    build.build_frontends()
    build.build_pybind()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        build.build_oracle()


_ensure_built()


@pytest.fixture(scope="session")
def gpu_available():
    import simpler_b200 as sb
    return sb.load().smp_device_count() > 0
