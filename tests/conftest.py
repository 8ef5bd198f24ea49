import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path against the oracle")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds libimbart and the oracle once per session when they are missing."""
    from imbatracer_b200 import build as B
    from oracle import oracle as O
    if not os.path.exists(B.lib_path()):
        B.build()
    if not os.path.exists(O.LIB):
        O.build()
    yield


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
