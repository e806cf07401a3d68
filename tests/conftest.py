import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def engine():
    from dpcrypto_b200 import Engine, build

    build.build()
    eng = Engine(0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def saber_tv():
    import numpy as np

    return dict(np.load(os.path.join(ROOT, "tests", "golden", "saber_l3_tv.npz")))
