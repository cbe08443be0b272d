import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 (B200) device")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_lib():
    """Builds (if stale) and loads libdiffsplat_b200.so; fails loudly without a GPU."""
    if not _has_gpu():
        pytest.fail("GPU test collected without a CUDA device")
    from diffsplat_b200 import build as B
    B.build()
    from diffsplat_b200 import _lib as L
    L.lib()
    assert L.lib().ds_device_check() == L.DS_OK, "not an sm_100 device"
    return L
