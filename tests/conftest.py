import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available():
    try:
        import torch  # noqa: F401  (only used to probe the device)
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def rbps():
    import rbps_b200
    rbps_b200.lib()
    return rbps_b200


@pytest.fixture(scope="session")
def ref():
    from oracle import ref as _ref
    if not _ref.available():
        pytest.skip("oracle library not built (make -C oracle)")
    return _ref
