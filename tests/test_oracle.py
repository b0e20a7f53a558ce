"""CPU checks of the oracle against the reference: golden vectors produced by
the reference's own compiled functions (tests/golden/make_golden.py), and,
where the reference build is present, live comparisons with it."""
import numpy as np
import pytest

import pyoracle as po
from conftest import GOLDEN_CASES


def _levels(golden, name):
    return int(golden[f"{name}_K"])


@pytest.mark.parametrize("name", list(GOLDEN_CASES))
def test_level_encode_matches_reference_golden(golden, name):
    """Predictor + quantizer + closed loop of every level, bit for bit."""
    f = golden[f"{name}_field"]
    K = _levels(golden, name)
    coarse = golden[f"{name}_coarsest"]
    for k in range(1, K + 1):
        s = 1 << (K - k)
        fine = np.ascontiguousarray(f[::s, ::s, ::s])
        q, u, c, dec = po.level_encode(fine, coarse, float(golden[f"{name}_L{k}_eb"]))
        assert np.array_equal(q.astype(np.uint16), golden[f"{name}_L{k}_codes"]), (name, k)
        assert np.array_equal(c, golden[f"{name}_L{k}_counts"])
        assert np.array_equal(u.view(np.uint8), golden[f"{name}_L{k}_unpred"].view(np.uint8))
        if k < K:
            # compressor-side grid equals the reference decoder's grid bit for bit
            assert np.array_equal(dec.view(np.uint8), golden[f"{name}_L{k}_decoded"].view(np.uint8))
        coarse = golden[f"{name}_L{k}_decoded"]


@pytest.mark.parametrize("name", list(GOLDEN_CASES))
def test_codec_matches_reference_golden(golden, name):
    """Whole container round trip: codes per stream and the decoded field equal
    the reference decoder's output on the same quant codes."""
    f = golden[f"{name}_field"]
    K = _levels(golden, name)
    ch, cl = GOLDEN_CASES[name]
    eb = float(golden[f"{name}_eb"])
    stream = po.compress(f, eb, chunk_high=ch, chunk_low=cl)
    for k in range(1, K + 1):
        dz, dy, dx = (np.array(f.shape) >> (K - k + 1))
        C = po.oracle().stzo_level_chunk(f.shape[2], f.shape[1], f.shape[0], k, ch, cl)
        for b in range(7):
            want = po.chunk_major(golden[f"{name}_L{k}_codes"][b], (dz, dy, dx), C)
            assert np.array_equal(po.stream_codes(stream, k, b), want), (name, k, b)
    out = po.decompress(stream)
    assert np.array_equal(out.view(np.uint8), golden[f"{name}_L{K}_decoded"].view(np.uint8))
    for lvl in range(1, K + 1):
        part = po.decompress(stream, lvl)
        want = golden[f"{name}_L{K - lvl}_decoded"] if lvl < K else golden[f"{name}_coarsest"]
        assert np.array_equal(part.view(np.uint8), want.view(np.uint8)), (name, lvl)


def test_planner_matches_reference_golden(golden):
    q, offs, rec = golden["plan_queries"], golden["plan_offsets"], golden["plan_records"]
    for i, row in enumerate(q):
        dims, ch, cl, a, b = row[:3], row[3], row[4], row[5:8], row[8:11]
        got = po.plan(dims, ch, cl, a, b)
        assert np.array_equal(got, rec[offs[i]:offs[i + 1]]), i


def test_error_bound_and_progressive_levels():
    from stz_b200 import fields

    f = fields.grf((64, 64, 64), 11.0 / 3.0, 3, np.float32)
    E = 1e-3 * (float(f.max()) - float(f.min()))
    eb = E / 8.2 * (1 - 1e-6)
    s = po.compress(f, eb)
    out = po.decompress(s)
    assert np.abs(out.astype(np.float64) - f).max() <= 8.2 * eb * (1 + 1e-6)
    half = po.decompress(s, 1)
    assert np.abs(half.astype(np.float64) - f[::2, ::2, ::2]).max() <= 2.7 * eb * (1 + 1e-5)


def test_box_equals_full_crop():
    from stz_b200 import fields

    f = fields.fronts((32, 32, 64), 4, np.float64)
    s = po.compress(f, 1e-4, chunk_high=8, chunk_low=4)
    full = po.decompress(s)
    for lo, hi in [((0, 0, 0), (63, 31, 31)), ((5, 7, 3), (40, 20, 30)), ((10, 0, 0), (10, 31, 31))]:
        box = po.decompress_box(s, lo, hi)
        sl = tuple(slice(min(a, b), max(a, b) + 1) for a, b in zip(lo[::-1], hi[::-1]))
        assert np.array_equal(box, full[sl])


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_matches_reference_live(dtype):
    rng = np.random.default_rng(9)
    for dims in [(7, 5, 3), (12, 8, 20), (2, 2, 2), (33, 17, 9)]:
        dz, dy, dx = dims
        fine = (rng.standard_normal((2 * dz, 2 * dy, 2 * dx)) * 10).astype(dtype)
        coarse = rng.standard_normal(dims).astype(dtype)
        for eb in (1e-1, 1e-5):
            a = po.level_encode(fine, coarse, eb)
            b = po.level_encode(fine, coarse, eb, use_ref=True)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
            assert np.array_equal(a[1].view(np.uint8), b[1].view(np.uint8))
            assert np.array_equal(a[3].view(np.uint8), b[3].view(np.uint8))


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", ["grf256_f32_1e-3", "fronts128x64x64_f64_1e-6"])
def test_oracle_stream_matches_reference_at_size(case):
    """The C restatement's whole-field codec against the reference's own level
    functions through the hierarchy (pyoracle.ref_round_trip): codes of every
    stream, the full decode and every progressive level, bit for bit. The
    256^3 GRF is the benchmark's 256^3 configuration at full size."""
    from stz_b200 import fields

    if case.startswith("grf"):
        f, rel = fields.grf((256, 256, 256), 11.0 / 3.0, 2025, np.float32), 1e-3
    else:
        f, rel = fields.fronts((64, 64, 128), 5, np.float64), 1e-6
    eb = po.pointwise_eb(f, rel)
    ref = po.ref_round_trip(f, eb)
    assert ref["closed_loop_ok"]
    stream = po.compress(f, eb)
    K = ref["K"]
    for k in range(1, K + 1):
        for b in range(7):
            assert np.array_equal(po.stream_codes(stream, k, b), ref["codes"][k - 1][b]), (k, b)
    u = np.uint64 if f.dtype == np.float64 else np.uint32
    assert np.array_equal(po.decompress(stream).view(u), ref["grids"][K].view(u))
    for lvl in range(1, K + 1):
        assert np.array_equal(po.decompress(stream, lvl).view(u), ref["grids"][K - lvl].view(u)), lvl
    if rel == 1e-6:
        assert sum(sum(c) for c in ref["unpred"]) > 0


@pytest.mark.skipif(not (po.ref_available() and po.rd_available()), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", ["grf64_f32_1e-3", "fronts64_f64_1e-6"])
def test_oracle_plain_pipeline_matches_reference(case):
    """The plain tricubic pipeline of src/float.cpp / src/double.cpp (stz-rd
    stencils, multipliers 1 / 2.5 / 6.25): the oracle's stream against the
    reference's functions through the hierarchy (pyoracle.ref_round_trip_plain)."""
    from stz_b200 import fields

    if case.startswith("grf"):
        f, rel = fields.grf((64, 64, 64), 11.0 / 3.0, 7, np.float32), 1e-3
    else:
        f, rel = fields.fronts((64, 64, 64), 3, np.float64), 1e-6
    mults = (1.0, 2.5, 6.25)
    eb = po.pointwise_eb(f, rel, mults)
    ref = po.ref_round_trip_plain(f, eb, mults)
    stream = po.compress(f, eb, predictor=1, mults=mults)
    K = ref["K"]
    for k in range(1, K + 1):
        for b in range(7):
            assert np.array_equal(po.stream_codes(stream, k, b), ref["codes"][k - 1][b]), (k, b)
    u = np.uint64 if f.dtype == np.float64 else np.uint32
    assert np.array_equal(po.decompress(stream).view(u), ref["grids"][K].view(u))
    if rel == 1e-6:
        assert sum(sum(c) for c in ref["unpred"]) > 0


@pytest.mark.skipif(not (po.ref_available() and po.dep_available()), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", ["grf64_1e-3", "logn64_1e-4", "ragged_112x80x48_1e-3", "fronts64_1e-6"])
def test_oracle_staged_pipeline_matches_reference(case):
    """The staged predictor of src/dependency.cpp (predictor 2, multipliers
    1 / 2.5 / 6.25): every level's codes of every block, and the full and
    progressive decodes of the oracle's stream, against the reference's
    stage functions in the reference's stage order
    (pyoracle.ref_round_trip_staged)."""
    from stz_b200 import fields

    if case.startswith("grf"):
        f, rel = fields.grf((64, 64, 64), 11.0 / 3.0, 7, np.float32), 1e-3
    elif case.startswith("logn"):
        f, rel = fields.lognormal((64, 64, 64), 5, np.float32), 1e-4
    elif case.startswith("fronts"):  # unpredictable values at this bound
        f, rel = fields.fronts((64, 64, 64), 3, np.float32), 1e-6
    else:
        f, rel = fields.grf((48, 80, 112), 3.0, 13, np.float32), 1e-3
    mults = (1.0, 2.5, 6.25)
    eb = po.pointwise_eb(f, rel, mults)
    ref = po.ref_round_trip_staged(f, eb, mults, chunk_high=8, chunk_low=4)
    stream = po.compress(f, eb, predictor=2, mults=mults, chunk_high=8, chunk_low=4)
    K = ref["K"]
    for k in range(1, K + 1):
        for b in range(7):
            assert np.array_equal(po.stream_codes(stream, k, b), ref["codes"][k - 1][b]), (k, b)
    out = po.decompress(stream)
    assert np.array_equal(out.view(np.uint32), ref["grids"][K].view(np.uint32))
    for lvl in range(1, K + 1):
        assert np.array_equal(po.decompress(stream, lvl).view(np.uint32), ref["grids"][K - lvl].view(np.uint32)), lvl
    # this eb carries no slack for the final rounding of dq + P in float
    # (the library's pointwise mode does): one ulp of the field's magnitude
    E = rel * (float(f.max()) - float(f.min())) + float(np.spacing(np.abs(f).max()))
    assert np.abs(out.astype(np.float64) - f).max() <= E
    if case.startswith("fronts"):
        assert sum(sum(c) for c in ref["unpred"]) > 0


def test_staged_pipeline_matches_reference_golden(golden):
    """The oracle's staged stream against golden codes and decode produced by
    src/dependency.cpp's stage functions (tests/golden/make_golden.py)."""
    f = golden["staged_field"]
    eb = float(golden["staged_eb"])
    K = int(golden["staged_K"])
    stream = po.compress(f, eb, predictor=2, mults=(1.0, 2.5, 6.25), chunk_high=8, chunk_low=4)
    for k in range(1, K + 1):
        want = golden[f"staged_L{k}_codes"]
        for b in range(7):
            assert np.array_equal(po.stream_codes(stream, k, b), want[b]), (k, b)
    assert np.array_equal(po.decompress(stream).view(np.uint32), golden["staged_decoded"].view(np.uint32))


@pytest.mark.skipif(not (po.ref_available() and po.stz2_available()), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("case", ["grf64_1e-3", "logn64_1e-4", "ragged_112x80x48_1e-3", "fronts64_1e-6"])
def test_oracle_truncated_pipeline_matches_reference(case):
    """The 12-point truncated bicubic predictor of src/stz2.cpp (predictor 3,
    one-axis interior cubic in double): codes and decodes of the oracle's
    stream against the reference's functions (pyoracle.ref_round_trip_trunc)."""
    from stz_b200 import fields

    if case.startswith("grf"):
        f, rel = fields.grf((64, 64, 64), 11.0 / 3.0, 7, np.float32), 1e-3
    elif case.startswith("logn"):
        f, rel = fields.lognormal((64, 64, 64), 5, np.float32), 1e-4
    elif case.startswith("fronts"):  # unpredictable values at this bound
        f, rel = fields.fronts((64, 64, 64), 3, np.float32), 1e-6
    else:
        f, rel = fields.grf((48, 80, 112), 3.0, 13, np.float32), 1e-3
    mults = (1.0, 2.5, 6.25)
    eb = po.pointwise_eb(f, rel, mults)
    ref = po.ref_round_trip_trunc(f, eb, mults, chunk_high=8, chunk_low=4)
    stream = po.compress(f, eb, predictor=3, mults=mults, chunk_high=8, chunk_low=4)
    K = ref["K"]
    for k in range(1, K + 1):
        for b in range(7):
            assert np.array_equal(po.stream_codes(stream, k, b), ref["codes"][k - 1][b]), (k, b)
    for lvl in range(0, K + 1):
        assert np.array_equal(po.decompress(stream, lvl).view(np.uint32), ref["grids"][K - lvl].view(np.uint32)), lvl
    if case.startswith("fronts"):
        assert sum(sum(c) for c in ref["unpred"]) > 0


def test_truncated_pipeline_matches_reference_golden(golden):
    """The oracle's predictor-3 stream against golden codes and decode made by
    src/stz2.cpp's functions (tests/golden/make_golden.py)."""
    f = golden["staged_field"]
    eb = float(golden["staged_eb"])
    K = int(golden["staged_K"])
    stream = po.compress(f, eb, predictor=3, mults=(1.0, 2.5, 6.25), chunk_high=8, chunk_low=4)
    for k in range(1, K + 1):
        want = golden[f"trunc_L{k}_codes"]
        for b in range(7):
            assert np.array_equal(po.stream_codes(stream, k, b), want[b]), (k, b)
    assert np.array_equal(po.decompress(stream).view(np.uint32), golden["trunc_decoded"].view(np.uint32))


def test_oracle_staged_f64_round_trip_and_box():
    """The staged predictor in double (the same expressions in T): bound,
    and boxes equal to the full decode's crop."""
    from stz_b200 import fields

    f = fields.fronts((64, 64, 64), 3, np.float64)
    mults = (1.0, 2.5, 6.25)
    eb = po.pointwise_eb(f, 1e-6, mults)
    stream = po.compress(f, eb, predictor=2, mults=mults)
    out = po.decompress(stream)
    assert np.abs(out - f).max() <= 1e-6 * (float(f.max()) - float(f.min())) + float(np.spacing(np.abs(f).max()))
    box = po.decompress_box(stream, (3, 5, 7), (40, 33, 20))
    assert np.array_equal(box.view(np.uint64), out[7:21, 5:34, 3:41].view(np.uint64))


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) not present")
def test_planner_matches_reference_live():
    rng = np.random.default_rng(17)
    for dims, ch, cl in [((128, 64, 64), 16, 8), ((64, 64, 64), 32, 16)]:
        for _ in range(300):
            a = rng.integers(-5, np.array(dims) + 5)
            b = rng.integers(-5, np.array(dims) + 5)
            assert np.array_equal(po.plan(dims, ch, cl, a, b), po.plan(dims, ch, cl, a, b, use_ref=True))


@pytest.mark.parametrize("suf", ["f32", "f64"])
def test_plain_cubic_predictor_matches_reference_golden(golden, suf):
    """Plain tricubic stencils of src/stz-rd.cpp (= src/float.cpp/double.cpp)."""
    ref, sub, diff = golden[f"plain_{suf}_ref"], golden[f"plain_{suf}_sub"], golden[f"plain_{suf}_diff"]
    dz, dy, dx = ref.shape
    fn = getattr(po.oracle(), "stzo_predict_plain_" + suf)
    for b in range(7):
        P = np.array([[[fn(b, po._p(ref), x, y, z, dx, dy, dz) for x in range(dx)] for y in range(dy)]
                      for z in range(dz)], dtype=ref.dtype)
        assert np.array_equal((sub - P).view(np.uint8), diff[b].view(np.uint8)), b


def test_plane_table_layouts_oracle():
    """Version-3 plane offsets and version-4 plane counts of either width
    decode alike in the oracle (the writer emits version 4, 2-byte counts
    here)."""
    from stream_tools import rewrite_plane_tables

    rng = np.random.default_rng(9)
    f = np.cumsum(rng.normal(0, 1, (64, 64, 64)), axis=2).astype(np.float32)
    b = po.compress(f, po.pointwise_eb(f, 1e-3))
    assert int.from_bytes(b[8:12], "little") == 4
    want = po.decompress(b)
    for v, w in ((3, 4), (4, 2), (4, 4)):
        got = po.decompress(rewrite_plane_tables(b, v, w))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (v, w)


def test_zstd_probe_rule():
    """Payload frames longer than 4 KiB are zstd-compressed only when zstd
    shrinks their first 4 KiB: Huffman payload of a noisy field is stored
    raw, while a field tiled from one small block (payload bytes repeat
    with the tile) keeps compressed payload frames. Stream headers are
    always tried."""
    from stream_tools import frame_sizes

    rng = np.random.default_rng(4)
    noisy = rng.normal(0, 1, (64, 64, 64)).astype(np.float32)
    fr = frame_sizes(po.compress(noisy, po.pointwise_eb(noisy, 1e-3)))
    big = [f for f in fr if f[2] == "payload" and f[4] > 4096]
    assert big and all(st == rw for _, _, _, st, rw in big)
    assert any(st < rw for _, _, kind, st, rw in fr if kind == "header")
    tile = rng.normal(0, 1, (8, 8, 64)).astype(np.float32)
    tiled = np.tile(tile, (8, 8, 1))
    fr = frame_sizes(po.compress(tiled, po.pointwise_eb(tiled, 1e-3)))
    assert any(st < rw for _, _, kind, st, rw in fr if kind == "payload" and rw > 4096)
