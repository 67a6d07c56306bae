import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "ar-renderer_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests against the oracle")
    config.addinivalue_line("markers", "slow: long-running statistical test")


def has_gpu() -> bool:
    try:
        from prgpu import abi

        return abi.gpu_lib().prgpu_list_devices(None, 0) >= 0 and _device_count() > 0
    except Exception:
        return False


def _device_count() -> int:
    import ctypes as C

    from prgpu import abi

    buf = (abi.DeviceInfo * 16)()
    return abi.gpu_lib().prgpu_list_devices(C.cast(buf, C.c_void_p), 16)


@pytest.fixture(scope="session")
def gpu():
    """The loaded CUDA module; GPU tests fail loudly (never skip) when it or the device is missing."""
    from prgpu import abi

    lib = abi.gpu_lib()
    assert _device_count() > 0, "no CUDA device visible to libprender_gpu.so"
    return lib


@pytest.fixture(scope="session")
def oracle():
    import ref

    if not ref.available():
        pytest.fail("oracle/_ref/libprref.so is missing: build it with `make -C oracle`")
    return ref
