import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "mls-mpm_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def native():
    from mls_mpm_b200 import load_library
    from mls_mpm_b200.build import build
    build()
    return load_library()


@pytest.fixture(scope="session")
def gpu(native):
    import ctypes
    n = ctypes.c_int()
    native.mpm_device_count(ctypes.byref(n))
    if n.value == 0:
        pytest.fail("GPU test selected but no CUDA device is visible")
    return native
