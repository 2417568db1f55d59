import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle_py
    oracle_py._load()
    return oracle_py


@pytest.fixture(scope="session")
def fsl():
    import fluam_b200
    from fluam_b200 import _lib
    _lib.load()
    return fluam_b200
