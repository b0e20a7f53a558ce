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


def random_model(rng, s_in=4.0, s_out=0.002, sh=(10, 10)):
    """A learned-correction record with random int8 weights (an untrained
    model: parity cases exercise the arithmetic, not the gain)."""
    import pyoracle as po

    m = po.Model()
    m.s_in, m.s_out = s_in, s_out
    w1 = rng.integers(-40, 41, (32, 16))
    w1[:, 14:] = 0
    for j in range(32):
        for i in range(16):
            m.w1[j][i] = int(w1[j, i])
        m.b1[j] = int(rng.integers(-400, 401))
        for i in range(32):
            m.w2[j][i] = int(rng.integers(-30, 31))
        m.b2[j] = int(rng.integers(-400, 401))
    for o in range(8):
        for i in range(32):
            m.w3[o][i] = int(rng.integers(-60, 61)) if o < 7 else 0
        m.b3[o] = int(rng.integers(-200, 201)) if o < 7 else 0
    m.m1, m.sh1, m.m2, m.sh2 = 200, int(sh[0]), 150, int(sh[1])
    return m


def model_file(records):
    """STZLMDL1 bytes of (second-finest, finest) records (None: absent)."""
    import pyoracle as po

    mask = (1 if records[0] is not None else 0) | (2 if records[1] is not None else 0)
    body = b"".join(po.model_record(r) for r in records if r is not None)
    return b"STZLMDL1" + np.uint32(mask).tobytes() + body
