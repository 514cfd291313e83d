import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the C-ABI library on the device")


@pytest.fixture(scope="session")
def ctx():
    import elmerfem_b200 as eg

    c = eg.Context(0)
    yield c
    c.close()
