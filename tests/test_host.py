"""CPU checks of the product library's host side: it loads, exports every
declared entry point, and its host logic (codebook, planner) agrees with the
oracle's independent implementation. No GPU calls."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyoracle as po
import stz_b200
from conftest import ROOT, random_model


def test_library_exports_every_declared_symbol():
    lib = stz_b200.load_library()
    names = set()
    inc = os.path.join(ROOT, "include")
    for dirpath, _, files in os.walk(inc):
        for fn in files:
            if fn.endswith(".h"):
                names |= set(re.findall(r"\b(stz_[a-z0-9_]+)\s*\(", open(os.path.join(dirpath, fn)).read()))
    assert names, "no declarations found"
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_library_has_no_oracle_dependency():
    with open(stz_b200.LIB_PATH, "rb") as f:
        blob = f.read()
    assert b"stzo_" not in blob and b"fd5ref_" not in blob


def test_default_opts_are_reference_defaults():
    o = stz_b200.default_opts()
    assert (o.mult_base, o.mult_low, o.mult_high) == (0.7, 2.7, 8.2)
    assert (o.radius, o.chunk_high, o.chunk_low, o.zstd_level) == (32768, 32, 16, 3)
    assert o.model is None and o.learned_flags == -1


def test_predictor_names_map_to_the_header_values():
    import stz_b200

    for name, v in (("dynamic", 0), ("cubic", 1), ("staged", 2), ("truncated", 3)):
        assert stz_b200.default_opts(predictor=name).predictor == v


def test_oracle_rejects_an_unknown_predictor():
    """A stream header naming a predictor past the four known ones does not
    decode (the library's parser rejects the same values)."""
    import pyoracle as po

    f = np.cumsum(np.random.default_rng(2).normal(0, 1, (64, 64, 64)), axis=2).astype(np.float32)
    b = bytearray(po.compress(f, po.pointwise_eb(f, 1e-3), predictor=3))
    assert int.from_bytes(b[16:20], "little") == 3  # magic, version, dtype, predictor
    po.decompress(bytes(b))
    b[16:20] = (4).to_bytes(4, "little")
    with pytest.raises(ValueError):
        po.decompress(bytes(b))


def test_struct_offsets_match_the_c_compiler(tmp_path):
    """Field offsets of the option / info structs as gcc lays them out."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "stz/stz.h"', "int main(void) {"]
    structs = (("stz_opts", stz_b200.Opts), ("stz_info", stz_b200.Info), ("stz_train_opts", stz_b200.TrainOpts),
               ("stz_train_stats", stz_b200.TrainStats))
    for struct, cls in structs:
        lines.append('printf("%%zu\\n", sizeof(%s));' % struct)
        for f, _ in cls._fields_:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (struct, f))
    lines.append("return 0; }")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for _, cls in structs:
        want.append(ctypes.sizeof(cls))
        want += [getattr(cls, f).offset for f, _ in cls._fields_]
    assert got == want


def _random_model_record(rng, s_in=4.0, s_out=0.05, sh=(9, 9)):
    return po.model_record(random_model(rng, s_in=s_in, s_out=s_out, sh=sh))


def test_model_bytes_round_trip_and_validation():
    rng = np.random.default_rng(11)
    r0, r1 = _random_model_record(rng), _random_model_record(rng)
    for mask, recs in ((1, [r0]), (2, [r1]), (3, [r0, r1])):
        data = b"STZLMDL1" + np.uint32(mask).tobytes() + b"".join(recs)
        m = stz_b200.Model.from_bytes(data)
        assert m.to_bytes() == data
    good = b"STZLMDL1" + np.uint32(3).tobytes() + r0 + r1
    bad_cases = [
        b"STZLMDL0" + good[8:],                              # magic
        good[:-1],                                           # truncated
        b"STZLMDL1" + np.uint32(0).tobytes(),                # empty mask
        b"STZLMDL1" + np.uint32(4).tobytes() + r0,           # unknown record bit
        b"STZLMDL1" + np.uint32(1).tobytes() + _random_model_record(rng, s_in=0.0),  # scale must be > 0
        b"STZLMDL1" + np.uint32(1).tobytes() + _random_model_record(rng, s_out=float("nan")),
        b"STZLMDL1" + np.uint32(2).tobytes() + _random_model_record(rng, sh=(0, 9)),  # shift out of range
        b"STZLMDL1" + np.uint32(2).tobytes() + _random_model_record(rng, sh=(9, 63)),
    ]
    for data in bad_cases:
        with pytest.raises(stz_b200.StzError) as e:
            stz_b200.Model.from_bytes(data)
        assert e.value.status == 5


def _hists():
    rng = np.random.default_rng(1)
    yield np.bincount(rng.geometric(0.3, 5000), minlength=64).astype(np.uint32)
    h = np.zeros(4096, np.uint32)
    h[2048] = 10**7
    h[2047] = h[2049] = 1000
    h[100] = 1
    yield h
    fib = [1, 1]
    while len(fib) < 40:
        fib.append(fib[-1] + fib[-2])
    yield np.array(fib, dtype=np.uint32)  # forces the length limit
    h = np.zeros(65536, np.uint32)
    h[32768] = 5
    yield h  # single symbol
    yield rng.integers(0, 3, 65536).astype(np.uint32)
    yield np.ones(3000, np.uint32)


def test_codebook_matches_oracle():
    for h in _hists():
        s1, l1 = stz_b200.codebook(h)
        s2, l2 = po.codebook(h)
        assert np.array_equal(s1, s2) and np.array_equal(l1, l2)
        assert l1.max() <= 24
        if len(l1) > 1:
            assert (2.0 ** -l1.astype(np.float64)).sum() <= 1.0  # Kraft


def test_run_slots_match_oracle():
    """Run-symbol slots: the highest window of unused codes, none when the
    range is full, sized by the plane (direct lengths up to 32, then powers
    of two)."""
    rng = np.random.default_rng(9)
    cases = []
    for nbins in (16, 64, 4096, 65536):
        for plane in (1, 2, 4, 16, 64, 256, 1024, 16384):
            h = np.zeros(nbins, np.uint32)
            h[nbins // 2] = 100
            cases.append((h.copy(), plane))                       # top free
            h[-3:] = 1
            cases.append((h.copy(), plane))                       # top used: next window down
            h2 = rng.integers(0, 3, nbins).astype(np.uint32)
            cases.append((h2, plane))                             # scattered free codes
            cases.append((np.ones(nbins, np.uint32), plane))      # none free
    for h, plane in cases:
        got = stz_b200.run_slots(h, plane)
        assert got == po.run_slots(h, plane), (len(h), plane)
        base, n = got
        if n:
            assert base >= 1 and base + n <= len(h) and not h[base:base + n].any()
    assert stz_b200.run_slots(np.zeros(65536, np.uint32), 1024) == (65536 - 36, 36)
    assert stz_b200.run_slots(np.zeros(65536, np.uint32), 64) == (65536 - 32, 32)
    assert stz_b200.run_slots(np.zeros(65536, np.uint32), 1) == (0, 0)


def test_codebook_is_optimal_without_length_limit():
    rng = np.random.default_rng(4)
    h = rng.integers(1, 1000, 300).astype(np.uint32)
    s, l = stz_b200.codebook(h)
    # Huffman cost equals the sum of merged weights
    import heapq

    heap = list(h.astype(np.int64))
    heapq.heapify(heap)
    cost = 0
    while len(heap) > 1:
        a, b = heapq.heappop(heap), heapq.heappop(heap)
        cost += a + b
        heapq.heappush(heap, a + b)
    assert int((h[s].astype(np.int64) * l).sum()) == cost


def test_planner_matches_oracle():
    rng = np.random.default_rng(2)
    for dims, ch, cl in [((256, 256, 256), 32, 16), ((384, 384, 256), 32, 16), ((64, 32, 128), 8, 4)]:
        for _ in range(200):
            a = rng.integers(-9, np.array(dims) + 9)
            b = rng.integers(-9, np.array(dims) + 9)
            if rng.random() < 0.25:
                ax = rng.integers(0, 3)
                b[ax] = a[ax]
            assert np.array_equal(stz_b200.plan_box(dims, ch, cl, a, b), po.plan(dims, ch, cl, a, b))


def test_planner_rejects_bad_dims():
    with pytest.raises(stz_b200.StzError) as e:
        stz_b200.plan_box((30, 32, 32), 8, 4, (0, 0, 0), (1, 1, 1))
    assert e.value.status == 2


def test_fields_generators():
    from stz_b200 import fields

    g = fields.grf((32, 32, 32), 3.0, 1)
    assert g.dtype == np.float32 and abs(float(g.mean())) < 1e-5 and abs(float(g.std()) - 1) < 1e-4
    ln = fields.lognormal((16, 16, 16), 1)
    assert (ln > 0).all()
    fr = fields.fronts((8, 8, 16), 1)
    assert fr.dtype == np.float64 and fr.shape == (8, 8, 16)


def test_ctypes_structs_match_header():
    """ctypes layouts agree with include/stz/stz.h (field order)."""
    hdr = open(os.path.join(ROOT, "include", "stz", "stz.h")).read()
    for struct, cls in (("stz_opts", stz_b200.Opts), ("stz_info", stz_b200.Info),
                        ("stz_server_opts", stz_b200.ServerOpts), ("stz_request", stz_b200.Request),
                        ("stz_result", stz_b200.Result), ("stz_server_stats", stz_b200.ServerStats)):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), hdr, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = re.findall(r"^\s*(?:const\s+)?(?:struct\s+\w+|u?int64_t|int|double|size_t|stz_status|void)\b\s*\**\s*"
                            r"([a-z0-9_, \[\]]+);", body, re.M)
        names = [re.sub(r"\[\d+\]", "", n).strip() for f in fields for n in f.split(",")]
        assert names == [f[0] for f in cls._fields_], struct
    # sizes that the C compiler and ctypes must agree on (x86-64 ABI)
    assert ctypes.sizeof(stz_b200.Request) == 4 + 4 + 24 + 24 + 4 + 4
    assert ctypes.sizeof(stz_b200.Result) == 4 + 4 + 8 + 24 + 8 + 8 + 8 + 8 + 4 + 4


def test_server_default_opts():
    lib = stz_b200.load_library()
    o = stz_b200.ServerOpts()
    lib.stz_server_default_opts(ctypes.byref(o))
    assert o.arena_bytes == 1 << 30 and o.max_batch == 64 and o.slots == 2 and o.autotune == 1
    assert o.fast_reserve == ctypes.c_size_t(-1).value  # a quarter of the arena
