"""The reference's experimental predictors on the GPU: the staged predictor
(STZ_PRED_STAGED, src/dependency.cpp) and the 12-point truncated bicubic
(STZ_PRED_TRUNCATED, src/stz2.cpp).

* Small fields: the GPU stream is byte for byte the oracle's (whose
  pipelines are themselves pinned to the reference's functions, CPU tests),
  and so are the full decode, every progressive level and boxes/slices.
* 256^3 f32 GRF: every level's codes of every block, the full decode and the
  progressive levels against the reference's own functions compiled from
  source (pyoracle.ref_round_trip_staged / ref_round_trip_trunc).
* 512^3 f32 lognormal (the benchmark field): pointwise bound, box = crop.
* What the modes refuse: the request server.
* dependency.cpp's stage functions at the function boundary."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MULTS = dict(mult_base=1.0, mult_low=2.5, mult_high=6.25)


def _bits(a):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


PRED_ID = {"staged": 2, "truncated": 3}


@pytest.mark.parametrize("pred", ["staged", "truncated"])
@pytest.mark.parametrize("case", ["grf64_f32", "fronts64_f64", "ragged_112x80x48_f32", "logn64_f32_1e-4"])
def test_stream_is_the_oracles(ctx, case, pred):
    from stz_b200 import fields

    chunks = {}
    if case == "grf64_f32":
        f, rel = fields.grf((64, 64, 64), 11.0 / 3.0, 7, np.float32), 1e-3
    elif case == "fronts64_f64":
        f, rel = fields.fronts((64, 64, 64), 3, np.float64), 1e-6
    elif case == "logn64_f32_1e-4":
        f, rel = fields.lognormal((64, 64, 64), 5, np.float32), 1e-4
    else:
        f, rel = fields.grf((48, 80, 112), 3.0, 13, np.float32), 1e-3
        chunks = dict(chunk_high=8, chunk_low=4)
    s = ctx.compress(f, eb=rel, eb_mode="rel", predictor=pred, **MULTS, **chunks)
    inf = s.info()
    assert inf.predictor == PRED_ID[pred]
    want = po.compress(f, inf.eb, predictor=PRED_ID[pred], mults=(1.0, 2.5, 6.25), **chunks)
    assert s.to_bytes() == want
    out = ctx.decompress(s)
    assert np.array_equal(_bits(out), _bits(po.decompress(want)))
    E = rel * (float(f.max()) - float(f.min()))
    assert np.abs(out.astype(np.float64) - f).max() <= E
    for lvl in range(1, inf.n_levels + 1):
        assert np.array_equal(_bits(ctx.decompress(s, level=lvl)), _bits(po.decompress(want, lvl))), lvl
    box = ctx.decompress_box(s, (3, 5, 7), (40, 33, 20))
    assert np.array_equal(_bits(box), _bits(out[7:21, 5:34, 3:41]))
    sl = ctx.decompress_box(s, (0, 9, 0), (f.shape[2] - 1, 9, f.shape[0] - 1))
    assert np.array_equal(_bits(sl).reshape(-1), _bits(out[:, 9:10, :]).reshape(-1))
    # a parsed copy decodes the same (header, plane tables, predictor field)
    assert np.array_equal(_bits(ctx.decompress(ctx.parse(s.to_bytes()))), _bits(out))


@pytest.mark.parametrize("pred", ["staged", "truncated"])
def test_256_matches_reference(ctx, pred):
    from stz_b200 import fields

    if not (po.ref_available() and po.dep_available() and po.stz2_available()):
        pytest.skip("oracle/_ref (the reference build) is missing")
    f = fields.grf((256, 256, 256), 11.0 / 3.0, 2025)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel", predictor=pred, **MULTS)
    inf = s.info()
    trip = po.ref_round_trip_staged if pred == "staged" else po.ref_round_trip_trunc
    ref = trip(f, inf.eb, inf.mults)
    K = ref["K"]
    for k in range(1, K + 1):
        for b in range(7):
            assert np.array_equal(ctx.stream_codes(s, k, b), ref["codes"][k - 1][b]), (k, b)
    out = ctx.decompress(s)
    assert np.array_equal(_bits(out), _bits(ref["grids"][K]))
    for lvl in range(1, K + 1):
        assert np.array_equal(_bits(ctx.decompress(s, level=lvl)), _bits(ref["grids"][K - lvl])), lvl
    assert np.abs(out.astype(np.float64) - f).max() <= 1e-3 * (float(f.max()) - float(f.min()))


@pytest.mark.parametrize("pred", ["staged", "truncated"])
def test_lognormal_512_bound_and_box(ctx, pred):
    from stz_b200 import fields

    f = fields.lognormal((512, 512, 512), 2025, np.float32, device="cuda:0")
    s = ctx.compress(f, eb=1e-3, eb_mode="rel", predictor=pred, **MULTS)
    out = torch.empty_like(f)
    ctx.decompress(s, out=out)
    E = 1e-3 * (float(f.max()) - float(f.min()))
    assert float((out.double() - f.double()).abs().max()) <= E
    box = ctx.decompress_box(s, (100, 37, 250), (227, 300, 261))
    assert np.array_equal(_bits(box), _bits(out[250:262, 37:301, 100:228]))
    # decoding again gives the same bits (the stages leave no state behind)
    out2 = torch.empty_like(f)
    ctx.decompress(s, out=out2)
    assert torch.equal(out.view(torch.int32), out2.view(torch.int32))


@pytest.mark.parametrize("pred", ["staged", "truncated"])
def test_server_refuses_the_stream(ctx, pred):
    from stz_b200 import Server, StzError, fields

    f = fields.grf((64, 64, 64), 11.0 / 3.0, 3, np.float32)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel", predictor=pred)
    with Server(0, arena_bytes=64 << 20, max_batch=8) as srv:
        with pytest.raises(StzError, match=pred):
            srv.add_stream(s.to_bytes())


@pytest.mark.parametrize("dims", [(9, 10, 12), (1, 2, 3), (4, 3, 5)])
def test_stage_functions_match_reference(ctx, dims):
    """stz_(de)preprocess_block_staged_dev against src/dependency.cpp's own
    preprocess_block / depreprocess_block / preprocess_block_staged /
    depreprocess_block_staged (oracle/_ref), every block, bit for bit, on
    random sub-blocks with a flat region, including axes of extent 1-3 where
    only the boundary forms run."""
    if not po.dep_available():
        pytest.skip("oracle/_ref (the reference build) is missing")
    import ctypes as C

    D = po.dep()
    rng = np.random.default_rng(sum(dims))
    dz, dy, dx = dims
    arrs = [rng.standard_normal(dims).astype(np.float32) for _ in range(9)]
    for a in arrs:
        a[: max(1, dz // 2)] = np.float32(1e-3)
    sub, coarse, rest = arrs[0], arrs[1], arrs[2:8]
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    refs_ptr = (C.c_void_p * 6)(*[r.ctypes.data for r in rest])
    for block in range(7):
        one_axis = block in (0, 1, 3)
        want = np.empty(dims, np.float32)
        back = np.empty(dims, np.float32)
        if one_axis:
            D.depref_preprocess_block(block, po._p(sub), po._p(coarse), po._p(want), dx, dy, dz)
            D.depref_depreprocess_block(block, po._p(want), po._p(coarse), po._p(back), dx, dy, dz)
            refs = [dev(coarse)]
        else:
            D.depref_preprocess_block_staged(block, po._p(sub), refs_ptr, po._p(want), dx, dy, dz)
            D.depref_depreprocess_block_staged(block, po._p(want), refs_ptr, po._p(back), dx, dy, dz)
            refs = [dev(r) for r in rest]
        sub_t, diff_t, out_t = dev(sub), torch.empty(dims, dtype=torch.float32, device="cuda"), None
        ctx.preprocess_block_staged(block, sub_t, refs, diff_t)
        out_t = torch.empty_like(diff_t)
        ctx.depreprocess_block_staged(block, diff_t, refs, out_t)
        ctx.sync()
        assert np.array_equal(_bits(diff_t), _bits(want)), block
        assert np.array_equal(_bits(out_t), _bits(back)), block
