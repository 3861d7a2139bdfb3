import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def reference_root():
    """The reference checkout the oracle's reference targets were built from: NNTC_REFERENCE_ROOT, else the tree
    oracle/Makefile recorded in oracle/_ref/REFERENCE_ROOT; None when neither names an existing tree (the tests that
    read reference files then skip)."""
    root = os.environ.get("NNTC_REFERENCE_ROOT")
    if not root:
        rec = os.path.join(ROOT, "oracle", "_ref", "REFERENCE_ROOT")
        if os.path.exists(rec):
            root = open(rec).read().strip()
    return root if root and os.path.isdir(root) else None


def reference_file(*parts):
    """A path inside the reference checkout, or a path that does not exist when there is none."""
    root = reference_root()
    return os.path.join(root, *parts) if root else os.path.join(ROOT, "_no_reference_", *parts)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built libnntc_b200.so")


def golden(name):
    import numpy as np

    return dict(np.load(os.path.join(ROOT, "tests", "golden", f"{name}.npz")))


@pytest.fixture(params=["t1_c0_2", "t2_c0_4"])
def case(request):
    return request.param, golden(request.param)
