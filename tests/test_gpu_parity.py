"""GPU parity: the sm_100a kernels, called through the C ABI, against the
reference's compiled functions (oracle/_ref), the plain-C oracle and the
golden vectors. Integer/byte results must be identical; floating-point
results are compared bit for bit as well (the reference is deterministic)."""
import numpy as np
import pytest

import pyoracle as po
import stz_b200
from conftest import GOLDEN_CASES

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def bits(a):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return a.view(np.uint8)


def tdt(dtype):
    return torch.float64 if np.dtype(dtype) == np.float64 else torch.float32


# ---- reference function boundary ------------------------------------------------
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [(20, 12, 8), (3, 5, 7), (2, 2, 2), (33, 16, 9)])
def test_block_kernels_match_reference(ctx, dtype, dims):
    """preprocess / depreprocess / to_full / ROI depreprocess, every block."""
    rng = np.random.default_rng(sum(dims))
    dz, dy, dx = dims
    ref = rng.standard_normal(dims).astype(dtype)
    ref[: dz // 2] = 0.001  # flat half: FTZ-sensitive blend weights
    sub = rng.standard_normal(dims).astype(dtype)
    use_ref = po.ref_available()
    R = po.ref() if use_ref else None
    suf = po._suf(dtype)
    tr, ts = torch.from_numpy(ref).cuda(), torch.from_numpy(sub).cuda()
    for block in range(7):
        for pred in (0, 1):
            # expected diff / reconstruction
            if pred == 0 and use_ref:
                diff = np.zeros(dims, dtype)
                getattr(R, "fd5ref_preprocess_block_zslab_" + suf)(block, po._p(sub), po._p(ref), po._p(diff), dx, dy,
                                                                    dz, 0, dz)
                rec = np.zeros(dims, dtype)
                getattr(R, "fd5ref_depreprocess_block_zslab_" + suf)(block, po._p(sub), po._p(ref), po._p(rec), dx, dy,
                                                                      dz, 0, dz)
                full = np.zeros((2 * dz, 2 * dy, 2 * dx), dtype)
                getattr(R, "fd5ref_depreprocess_block_zslab_to_full_" + suf)(block, po._p(sub), po._p(ref),
                                                                             po._p(full), dx, dy, dz, 0, dz)
            else:
                fn = getattr(po.oracle(), ("stzo_predict_plain_" if pred else "stzo_predict_") + suf)
                P = np.array([[[fn(block, po._p(ref), x, y, z, dx, dy, dz) for x in range(dx)] for y in range(dy)]
                              for z in range(dz)], dtype=dtype)
                diff, rec = sub - P, sub + P
                full = np.zeros((2 * dz, 2 * dy, 2 * dx), dtype)
                s = block + 1
                full[(s >> 2) & 1::2, (s >> 1) & 1::2, s & 1::2] = rec
            out = torch.zeros_like(tr)
            ctx.preprocess_block(block, ts, tr, out, predictor=pred)
            assert np.array_equal(bits(out), bits(diff)), ("pre", block, pred)
            out.zero_()
            ctx.depreprocess_block(block, ts, tr, out, predictor=pred)
            assert np.array_equal(bits(out), bits(rec)), ("de", block, pred)
            fo = torch.zeros((2 * dz, 2 * dy, 2 * dx), dtype=tr.dtype, device="cuda")
            ctx.depreprocess_block_to_full(block, ts, tr, fo, predictor=pred)
            assert np.array_equal(bits(fo), bits(full)), ("full", block, pred)
            # ROI sub-range (FD5:978-999): only the range is written
            out.fill_(7)
            s0, e0 = (1, 0, 1), (dx, max(1, dy - 1), dz)
            ctx.depreprocess_block_roi(block, ts, tr, out, e0, s0, predictor=pred)
            want = np.full(dims, 7, dtype)
            want[s0[2]:e0[2], s0[1]:e0[1], s0[0]:e0[0]] = rec[s0[2]:e0[2], s0[1]:e0[1], s0[0]:e0[0]]
            assert np.array_equal(bits(out), bits(want)), ("roi", block, pred)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_quantize_dequantize_match_reference(ctx, dtype):
    rng = np.random.default_rng(3)
    d = (rng.standard_normal(100003) * rng.choice([1e-3, 1, 1e4], 100003)).astype(dtype)
    d[:5] = [0.0, -0.0, np.inf, -np.inf, np.nan]
    eb, radius = 1e-2, 32768
    if po.ref_available():
        q_ref = np.zeros(d.size, np.int32)
        u_ref = np.zeros(d.size, dtype)
        nu = getattr(po.ref(), "fd5ref_quantize_range_nodec_" + po._suf(dtype))(po._p(d), d.size, eb, radius,
                                                                                  po._p(q_ref), po._p(u_ref), d.size)
    else:
        q_ref = np.zeros(d.size, np.int32)
        u_ref = np.zeros(d.size, dtype)
        nu = getattr(po.oracle(), "stzo_quantize_" + po._suf(dtype))(po._p(d), d.size, eb, radius, po._p(q_ref),
                                                                      po._p(u_ref), d.size)
    td = torch.from_numpy(d).cuda()
    q = torch.zeros(d.size, dtype=torch.int32, device="cuda")
    u = torch.zeros(d.size, dtype=td.dtype, device="cuda")
    n = ctx.quantize(td, eb, radius, q, u)
    assert n == nu > 0
    assert np.array_equal(q.cpu().numpy(), q_ref)
    assert np.array_equal(bits(u[:n]), bits(u_ref[:nu]))
    out = torch.zeros_like(td)
    ctx.dequantize(q, eb, radius, u, out)
    want = po.ref_dequantize(q_ref, eb, radius, u_ref[:nu], dtype) if po.ref_available() else None
    if want is not None:
        assert np.array_equal(bits(out), bits(want))
    fin = np.isfinite(d)
    assert np.abs(out.cpu().numpy()[fin].astype(np.float64) - d[fin]).max() <= eb * (1 + 1e-6)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_split_merge_match_reference(ctx, dtype):
    rng = np.random.default_rng(5)
    f = rng.standard_normal((12, 10, 16)).astype(dtype)
    subs = np.zeros((8, 6, 5, 8), dtype)
    if po.ref_available():
        getattr(po.ref(), "fd5ref_slice_full_data_" + po._suf(dtype))(po._p(f), po._p(subs), 16, 10, 12)
    else:
        for s in range(8):
            subs[s] = f[(s >> 2) & 1::2, (s >> 1) & 1::2, s & 1::2]
    tf = torch.from_numpy(f).cuda()
    ts = torch.zeros((8, 6, 5, 8), dtype=tf.dtype, device="cuda")
    ctx.split(tf, ts)
    assert np.array_equal(bits(ts), bits(subs))
    back = torch.zeros_like(tf)
    ctx.merge(ts, back)
    assert np.array_equal(bits(back), bits(f))


# ---- whole codec vs golden vectors -------------------------------------------
@pytest.mark.parametrize("name", list(GOLDEN_CASES))
def test_codec_matches_reference_golden(ctx, golden, name):
    f = golden[f"{name}_field"]
    K = int(golden[f"{name}_K"])
    ch, cl = GOLDEN_CASES[name]
    eb = float(golden[f"{name}_eb"])
    s = ctx.compress(f, eb=eb, eb_mode="abs", bound_mode="reference", chunk_high=ch, chunk_low=cl)
    assert s.info().eb == eb
    for k in range(1, K + 1):
        dz, dy, dx = np.array(f.shape) >> (K - k + 1)
        C = po.oracle().stzo_level_chunk(f.shape[2], f.shape[1], f.shape[0], k, ch, cl)
        for b in range(7):
            want = po.chunk_major(golden[f"{name}_L{k}_codes"][b], (dz, dy, dx), C)
            assert np.array_equal(ctx.stream_codes(s, k, b), want), (k, b)
    out = ctx.decompress(s)
    assert np.array_equal(bits(out), bits(golden[f"{name}_L{K}_decoded"]))
    for lvl in range(1, K + 1):
        want = golden[f"{name}_L{K - lvl}_decoded"] if lvl < K else golden[f"{name}_coarsest"]
        assert np.array_equal(bits(ctx.decompress(s, level=lvl)), bits(want)), lvl
    # the stream itself equals the oracle's byte for byte
    assert s.to_bytes() == po.compress(f, eb, chunk_high=ch, chunk_low=cl)


# ---- whole codec vs the oracle ----------------------------------------------------
CASES = [
    # (generator, shape, dtype, rel, predictor, chunks, zstd)
    ("grf", (64, 64, 64), np.float32, 1e-3, 0, (32, 16), 3),
    ("grf", (64, 64, 64), np.float32, 1e-3, 1, (32, 16), 3),
    ("logn", (64, 64, 128), np.float32, 1e-4, 0, (16, 8), 3),
    ("fronts", (32, 48, 64), np.float64, 1e-6, 0, (8, 4), 3),
    ("fronts", (32, 48, 64), np.float64, 1e-3, 1, (8, 4), 0),
    ("grf", (16, 16, 16), np.float32, 1e-2, 0, (8, 4), 1),
    ("grf", (128, 64, 32), np.float32, 1e-5, 0, (16, 8), 3),
]


def make_field(gen, shape, dtype, seed):
    from stz_b200 import fields

    if gen == "grf":
        return fields.grf(shape, 11.0 / 3.0, seed, dtype)
    if gen == "logn":
        return fields.lognormal(shape, seed, dtype)
    return fields.fronts(shape, seed, dtype)


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}-{np.dtype(c[2]).name}-{c[3]}-p{c[4]}" for c in CASES])
def test_stream_and_decode_match_oracle(ctx, case):
    gen, shape, dtype, rel, pred, (ch, cl), zl = case
    f = make_field(gen, shape, dtype, 21)
    s = ctx.compress(f, eb=rel, eb_mode="rel", predictor=pred, chunk_high=ch, chunk_low=cl, zstd_level=zl)
    inf = s.info()
    ref_bytes = po.compress(f, inf.eb, predictor=pred, chunk_high=ch, chunk_low=cl, zstd_level=zl)
    assert s.to_bytes() == ref_bytes
    out = ctx.decompress(s)
    assert np.array_equal(bits(out), bits(po.decompress(ref_bytes)))
    E = rel * (float(f.max()) - float(f.min()))
    assert np.abs(out.astype(np.float64) - f.astype(np.float64)).max() <= E  # pointwise bound, FP64
    for lvl in (1, 2):
        assert np.array_equal(bits(ctx.decompress(s, level=lvl)), bits(po.decompress(ref_bytes, lvl)))
    # a parsed copy decodes the same
    s2 = ctx.parse(ref_bytes)
    assert np.array_equal(bits(ctx.decompress(s2)), bits(out))


@pytest.mark.parametrize("rel", [3e-6, 1e-4])
def test_wide_codebooks_decode_exactly(ctx, rel):
    """White noise at a tight bound: thousands of distinct codes, many longer
    than the decoder's table (the canonical long-code search and its shared
    and global symbol tails), plus unpredictable values at 3e-6."""
    rng = np.random.default_rng(77)
    f = rng.uniform(-1, 1, (64, 64, 64)).astype(np.float32)
    s = ctx.compress(f, eb=rel, eb_mode="rel", chunk_high=16, chunk_low=8)
    b = s.to_bytes()
    assert b == po.compress(f, s.info().eb, chunk_high=16, chunk_low=8)
    K = s.info().n_levels
    # the finest streams use > 7000 symbols, > 6000 of them with codes longer than 12 bits
    assert max(len(np.unique(po.stream_codes(b, K, blk))) for blk in range(7)) > 7000
    out = ctx.decompress(s)
    assert np.array_equal(bits(out), bits(po.decompress(b)))
    box = ctx.decompress_box(s, (5, 9, 13), (50, 40, 60))
    assert np.array_equal(bits(box), bits(out[13:61, 9:41, 5:51]))


def test_reference_bound_mode_matches_cli_semantics(ctx):
    f = make_field("grf", (32, 32, 32), np.float32, 2)
    s = ctx.compress(f, eb=1e-3, eb_mode="abs", bound_mode="reference", chunk_high=8, chunk_low=4)
    inf = s.info()
    assert inf.eb == 1e-3 and abs(inf.max_error - 8.2e-3) < 1e-12
    out = ctx.decompress(s)
    assert np.abs(out.astype(np.float64) - f).max() <= 8.2e-3 * (1 + 1e-4)


# ---- random access -----------------------------------------------------------------
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_box_and_slice_equal_full_decode(ctx, dtype):
    f = make_field("fronts", (64, 64, 128), dtype, 8)
    s = ctx.compress(f, eb=1e-4, eb_mode="rel", chunk_high=16, chunk_low=8)
    full = ctx.decompress(s)
    rng = np.random.default_rng(1)
    queries = [((0, 0, 0), (63, 63, 63)), ((127, 63, 63), (0, 0, 0)), ((5, 9, 2), (5, 60, 40)),
               ((0, 31, 0), (127, 31, 63)), ((100, 50, 20), (100, 50, 20)), ((-10, -3, 5), (300, 2, 5))]
    for _ in range(12):
        a = rng.integers(0, [128, 64, 64])
        b = a + rng.integers(0, 40, 3)
        queries.append((tuple(a), tuple(b)))
    bytes_ = s.to_bytes()
    for lo, hi in queries:
        box = ctx.decompress_box(s, lo, hi)
        sl = []
        for ax, n in zip((2, 1, 0), (64, 64, 128)):
            a_, b_ = lo[ax], hi[ax]
            if a_ == b_:
                v = max(0, min(a_, n - 1))
                sl.append(slice(v, v + 1))
            else:
                sl.append(slice(max(0, min(a_, b_)), min(n - 1, max(a_, b_)) + 1))
        assert np.array_equal(bits(box), bits(full[tuple(sl)])), (lo, hi)
        assert np.array_equal(bits(box), bits(po.decompress_box(bytes_, lo, hi)))


def test_resident_stream_decodes_identically(ctx):
    f = make_field("grf", (64, 64, 64), np.float32, 4)
    s = ctx.compress(f, eb=1e-3)
    before = ctx.decompress(s)
    ctx.upload(s)
    assert np.array_equal(bits(ctx.decompress(s)), bits(before))
    assert np.array_equal(bits(ctx.decompress(s, level=1)), bits(po.decompress(s.to_bytes(), 1)))
    box = ctx.decompress_box(s, (3, 4, 5), (40, 41, 42))
    assert np.array_equal(bits(box), bits(before[5:43, 4:42, 3:41]))


def test_device_pointer_paths(ctx):
    f = make_field("grf", (64, 64, 64), np.float32, 6)
    tf = torch.from_numpy(f).cuda()
    s = ctx.compress(tf, eb=1e-3)
    assert s.to_bytes() == ctx.compress(f, eb=1e-3).to_bytes()
    out = torch.empty_like(tf)
    ctx.decompress(s, out=out)
    assert np.array_equal(bits(out), bits(po.decompress(s.to_bytes())))
    box = torch.empty((10, 20, 30), dtype=torch.float32, device="cuda")
    ctx.decompress_box(s, (1, 2, 3), (30, 21, 12), out=box)
    assert np.array_equal(bits(box), bits(out[3:13, 2:22, 1:31]))


# ---- errors are reported, not hidden ------------------------------------------------
def test_errors(ctx):
    f = np.zeros((30, 32, 32), np.float32)
    with pytest.raises(stz_b200.StzError) as e:
        ctx.compress(f, eb=1e-3)
    assert e.value.status == 2
    g = make_field("grf", (32, 32, 32), np.float32, 1)
    with pytest.raises(stz_b200.StzError) as e:
        ctx.compress(g, eb=1e-3, chunk_high=32)  # 16 % 32 != 0
    assert e.value.status == 2
    with pytest.raises(stz_b200.StzError):
        ctx.compress(g, eb=-1.0)
    s = ctx.compress(g, eb=1e-3, chunk_high=8, chunk_low=4)
    with pytest.raises(stz_b200.StzError) as e:
        ctx.decompress(s, level=9)
    assert e.value.status == 7
    b = bytearray(s.to_bytes())
    with pytest.raises(stz_b200.StzError):
        ctx.parse(bytes(b[:100]))
    b[0] ^= 0xFF
    with pytest.raises(stz_b200.StzError):
        ctx.parse(bytes(b))
    # corrupt a payload byte: decodes to wrong values or reports an error, never faults
    b = bytearray(s.to_bytes())
    b[-5] ^= 0x5A
    try:
        s3 = ctx.parse(bytes(b))
        ctx.decompress(s3)
    except stz_b200.StzError:
        pass
    ctx.sync()


@pytest.mark.parametrize("suf", ["f32", "f64"])
def test_plain_cubic_kernel_matches_reference_golden(ctx, golden, suf):
    ref, sub, diff = golden[f"plain_{suf}_ref"], golden[f"plain_{suf}_sub"], golden[f"plain_{suf}_diff"]
    tr, ts = torch.from_numpy(ref).cuda(), torch.from_numpy(sub).cuda()
    for b in range(7):
        out = torch.zeros_like(tr)
        ctx.preprocess_block(b, ts, tr, out, predictor=1)
        assert np.array_equal(bits(out), bits(diff[b])), b


# ---- run symbols (container version 3 and later) ---------------------------------
@pytest.mark.parametrize("case", ["constant", "noise_full_range", "ramp_spikes", "tiny_chunks"])
def test_run_symbol_streams_match_oracle(ctx, case):
    """Streams whose planes are one long run (single-symbol codebooks of run
    symbols), streams whose code range is full (no free window: no runs),
    mixed runs and spikes, and planes of 4 codes (2x2 chunks)."""
    rng = np.random.default_rng(3)
    kw = dict(chunk_high=8, chunk_low=4)
    if case == "constant":
        f = np.full((32, 32, 64), 2.5, np.float32)
        rel, radius = 1e-3, 32768
    elif case == "noise_full_range":
        f = rng.uniform(-1, 1, (32, 32, 32)).astype(np.float32)
        rel, radius = 1e-4, 64
    elif case == "ramp_spikes":
        f = np.fromfunction(lambda z, y, x: 0.01 * x + 0.003 * y * z, (64, 32, 32), dtype=np.float32)
        idx = rng.integers(0, f.size, 300)
        f.flat[idx] += rng.normal(0, 5, 300).astype(np.float32)
        rel, radius = 1e-4, 256
    else:
        f = make_field("grf", (16, 16, 32), np.float32, 4)
        rel, radius = 1e-3, 32768
        kw = dict(chunk_high=2, chunk_low=1)
    s = ctx.compress(f, eb=rel, eb_mode="rel", radius=radius, **kw)
    b = s.to_bytes()
    assert int.from_bytes(b[8:12], "little") == 4
    assert b == po.compress(f, s.info().eb, radius=radius, **kw)
    out = ctx.decompress(s)
    assert np.array_equal(bits(out), bits(po.decompress(b)))
    E = rel * max(float(f.max()) - float(f.min()), 0.0) or rel
    assert np.abs(out.astype(np.float64) - f).max() <= E
    nz, ny, nx = f.shape
    for lo, hi in (((1, 2, 3), (nx - 3, ny - 2, nz - 1)), ((0, ny // 2, 0), (nx - 1, ny // 2, nz - 1))):
        box = ctx.decompress_box(s, lo, hi)
        want = out[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        assert np.array_equal(bits(box), bits(want)), (lo, hi)


# ---- plane tables (container version 4) ----------------------------------------------
def test_plane_table_layouts_decode_alike(ctx):
    """The same stream with its plane tables as version-3 offsets, version-4
    2-byte counts (what the writer chose) and version-4 4-byte counts decodes
    to the same field, full and as a box."""
    from stream_tools import rewrite_plane_tables

    f = make_field("grf", (64, 64, 64), np.float32, 11)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel")
    b = s.to_bytes()
    assert b == po.compress(f, s.info().eb)
    want = ctx.decompress(s)
    lo, hi = (5, 9, 13), (40, 33, 50)
    wbox = ctx.decompress_box(s, lo, hi)
    for v, w in ((3, 4), (4, 4)):
        b2 = rewrite_plane_tables(b, v, w)
        s2 = ctx.parse(b2)
        assert np.array_equal(bits(ctx.decompress(s2)), bits(want)), (v, w)
        assert np.array_equal(bits(ctx.decompress_box(s2, lo, hi)), bits(wbox)), (v, w)


def test_wide_planes_use_four_byte_counts(ctx):
    """128^3 marker chunks of noise: planes of 16384 codes need more than
    65535 bits, so the writer stores 4-byte plane counts; the stream is the
    oracle's and decodes to it."""
    rng = np.random.default_rng(5)
    f = rng.normal(0, 1, (256, 256, 256)).astype(np.float32)
    kw = dict(chunk_high=128, chunk_low=16)
    s = ctx.compress(f, eb=1e-4, eb_mode="rel", **kw)
    b = s.to_bytes()
    assert b == po.compress(f, s.info().eb, **kw)
    out = ctx.decompress(s)
    assert np.array_equal(bits(out), bits(po.decompress(b)))
