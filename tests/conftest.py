import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle (CPU checker) and libsynx.so in-tree if they are missing."""
    import oracle as O
    if not os.path.exists(O.LIB_PATH):
        O.build()
    from ants_b200 import build
    if not os.path.exists(build.LIB):
        build.build_lib()
    yield


@pytest.fixture(scope="session")
def cuda():
    if not _cuda_available():
        pytest.fail("GPU test collected without a CUDA device")
    import torch
    torch.cuda.init()
    return torch.device("cuda:0")
