import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the native library")
    config.addinivalue_line("markers", "slow: larger GPU cases")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def native():
    import compressiontests_b200 as cb
    cb.load()
    return cb


@pytest.fixture(scope="session")
def ctx(native):
    c = native.CudaContext(0)
    yield c
    c.close()


@pytest.fixture
def rng():
    return np.random.default_rng(20261203)
