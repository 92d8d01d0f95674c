import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libsteel_b200.so")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def steel():
    """The CUDA library; building it is the test setup, a missing GPU is a failure, not a skip."""
    from steel_webgpu_b200 import build as b
    b.build()
    import steel_webgpu_b200 as sw
    return sw
