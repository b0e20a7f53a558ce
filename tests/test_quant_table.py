"""CPU check of the plain f32 level encoder's quantizer table: the device's
table decision, emulated here with float32 arithmetic, gives the reference
quantizer's code (quantize_range_nodec, FD5:1216-1229, through the oracle)
for residuals at, around and between every threshold of the table, for
several error bounds and both signs."""
import ctypes as C

import numpy as np
import pytest

import pyoracle as po
import stz_b200


def _oracle_codes(d, eb, radius):
    q = np.zeros(d.size, np.int32)
    u = np.zeros(d.size, np.float32)
    po.oracle().stzo_quantize_f32(d.ctypes.data_as(C.c_void_p), d.size, eb, radius, q.ctypes.data_as(C.c_void_p),
                                  u.ctypes.data_as(C.c_void_p), u.size)
    return q


def _table_codes(d, tab, r2, radius):
    """The device's quantize_table, with None where it defers to
    quantize_full (outside the entry's interval)."""
    a = np.abs(d).astype(np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        h = np.rint(a * r2)
    h = np.clip(np.nan_to_num(h, nan=0.0, posinf=1e9), 0, 63).astype(np.int64)
    e = tab[h]
    inside = (a >= e[:, 0]) & (a < e[:, 1])
    ok = (a >= e[:, 2]) & (a <= e[:, 3])
    code = np.where(ok, np.where(d < 0, radius - h, radius + h), 0)
    return code, inside


@pytest.mark.parametrize("eb,radius", [(1e-3, 32768), (3.3e-5, 32768), (0.0123, 512), (7.7e-9, 32768), (2.5, 32768)])
def test_quant_table_matches_reference_quantizer(eb, radius):
    tab, r2, on = stz_b200.quant_table(eb, radius)
    assert on
    f32 = np.float32
    pts = [np.float32(0), np.float32(1e-40)]
    for h in range(64):
        for v in tab[h]:
            if np.isfinite(v):
                v = f32(v)
                for k in range(-3, 4):
                    x = v
                    for _ in range(abs(k)):
                        x = np.nextafter(x, f32(np.inf) if k > 0 else f32(0))
                    pts.append(x)
    rng = np.random.default_rng(5)
    pts = np.array(pts, np.float32)
    rnd = (rng.random(200000) * 140 * eb).astype(np.float32)
    d = np.concatenate([pts, -pts, rnd, -rnd]).astype(np.float32)
    want = _oracle_codes(d, eb, radius)
    code, inside = _table_codes(d, tab, r2, radius)
    assert inside.mean() > 0.5
    bad = inside & (code != want)
    assert not bad.any(), (d[bad][:5], code[bad][:5], want[bad][:5])
