import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built libnntc_b200.so")


def golden(name):
    import numpy as np

    return dict(np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz")))


@pytest.fixture(params=["t1_c0_2", "t2_c0_4"])
def case(request):
    return request.param, golden(request.param)
