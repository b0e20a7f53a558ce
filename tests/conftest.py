import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "sc25-stz2_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "fd5_golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on a B200)")


def _ensure_built():
    import pyoracle

    if not os.path.exists(pyoracle.ORACLE_SO):
        pyoracle.build(ref=False)
    from importlib import import_module

    b = import_module("build")  # sc25-stz2_b200/build.py
    b.build()


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def ctx():
    from stz_b200 import Context

    c = Context(0)
    yield c
    c.close()


GOLDEN_CASES = {
    # name: (chunk_high, chunk_low) compatible with the case's dims
    "grf32": (8, 4),
    "logn32": (8, 4),
    "fronts64": (4, 2),
    "flat32": (8, 4),
}
