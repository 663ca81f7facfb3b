import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    """This project's C restatement of the golden model (the checker)."""
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def lib():
    """The product library (C ABI); built in-tree if missing."""
    from anechoic_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from anechoic_b200 import build_ext
        build_ext.build()
    return _lib.load()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
