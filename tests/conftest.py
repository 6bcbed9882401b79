import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libsfgpu.so")


@pytest.fixture(scope="session")
def gpu_lib():
    """The built CUDA library; GPU tests fail (not skip) when it is missing."""
    from field_b200 import _native
    lib = _native.load()
    n = __import__("ctypes").c_int()
    rc = lib.sfgpu_device_count(__import__("ctypes").byref(n))
    assert rc == 0 and n.value > 0, "no CUDA device visible to libsfgpu"
    return lib
