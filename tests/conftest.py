import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def o64():
    from oracle import Oracle
    return Oracle("f64")


@pytest.fixture(scope="session")
def o32():
    from oracle import Oracle
    return Oracle("f32")


@pytest.fixture(scope="session")
def rt():
    import iqm_b200
    r = iqm_b200.Runtime(0)
    yield r
    r.close()
