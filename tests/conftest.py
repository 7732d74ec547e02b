import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def restatement():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference():
    import oracle
    if not oracle.reference_available():
        pytest.skip("reference build (oracle/_ref) not present on this machine")
    return oracle.Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcons_b200 import _lib
    _lib.lib()
    return torch.device("cuda:0")
