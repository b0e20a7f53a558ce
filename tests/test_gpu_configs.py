"""The benchmark configurations at full size, against the oracle and through
size-independent properties:

* 256^3 f32 GRF k^-11/3, rel eb 1e-3: stream byte-identical to the oracle's,
  decode bit-exact;
* 512^3 f32 lognormal exp(1.5 g), rel eb 1e-2 / 1e-3 / 1e-4: max |x - x'| <= E
  in FP64, progressive levels 1-3 equal to the full decode's strided samples,
  a parsed copy decodes identically; at 1e-3 the stream is the oracle's;
* 384x384x256 f64 GRF k^-5/3 + 20 tanh fronts, rel eb 1e-6 / 1e-3: 100 random
  boxes (edges uniform in [16, 128]) and 20 axis-aligned slices equal to the
  full decode, and the bound."""
import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def u(a):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def test_grf_256_stream_is_the_oracles(ctx):
    from stz_b200 import fields

    f = fields.grf((256, 256, 256), 11.0 / 3.0, 2025)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel")
    b = s.to_bytes()
    assert b == po.compress(f, s.info().eb)
    out = ctx.decompress(s)
    assert np.array_equal(u(out), u(po.decompress(b)))
    E = 1e-3 * (float(f.max()) - float(f.min()))
    assert np.abs(out.astype(np.float64) - f).max() <= E


@pytest.mark.parametrize("rel", [1e-2, 1e-3, 1e-4])
def test_lognormal_512(ctx, rel):
    from stz_b200 import fields

    f = fields.lognormal((512, 512, 512), 2025, np.float32, device="cuda:0")
    s = ctx.compress(f, eb=rel, eb_mode="rel")
    out = torch.empty_like(f)
    ctx.decompress(s, out=out)
    E = rel * (float(f.max()) - float(f.min()))
    assert float((out.double() - f.double()).abs().max()) <= E
    for lvl in (1, 2, 3):
        st = 1 << lvl
        got = torch.from_numpy(ctx.decompress(s, level=lvl)).cuda()
        assert torch.equal(got.view(torch.int32), out[::st, ::st, ::st].contiguous().view(torch.int32)), lvl
    b = s.to_bytes()
    s2 = ctx.parse(b)
    out2 = torch.empty_like(f)
    ctx.decompress(s2, out=out2)
    assert torch.equal(out2.view(torch.int32), out.view(torch.int32))
    if rel == 1e-3:
        fh = f.cpu().numpy()
        ref = po.compress(fh, s.info().eb)
        assert b == ref
        assert np.array_equal(u(out), u(po.decompress(ref)))


@pytest.mark.parametrize("rel", [1e-6, 1e-3])
def test_fronts_384_boxes_and_slices(ctx, rel):
    from stz_b200 import fields

    nz, ny, nx = 256, 384, 384
    f = fields.fronts((nz, ny, nx), 31, np.float64, device="cuda:0")
    s = ctx.compress(f, eb=rel, eb_mode="rel")
    full = torch.empty_like(f)
    ctx.decompress(s, out=full)
    E = rel * (float(f.max()) - float(f.min()))
    assert float((full - f).abs().max()) <= E
    rng = np.random.default_rng(int(1 / rel) % 1000)
    dims = (nx, ny, nz)
    reqs = []
    for _ in range(100):
        e = rng.integers(16, 129, 3)
        lo = [int(rng.integers(0, d - x + 1)) for d, x in zip(dims, e)]
        reqs.append((lo, [a + int(x) - 1 for a, x in zip(lo, e)]))
    for _ in range(20):
        ax = int(rng.integers(0, 3))
        lo, hi = [0, 0, 0], [d - 1 for d in dims]
        lo[ax] = hi[ax] = int(rng.integers(0, dims[ax]))
        reqs.append((lo, hi))
    for lo, hi in reqs:
        box = torch.empty((hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1), dtype=f.dtype, device="cuda")
        ctx.decompress_box(s, lo, hi, out=box)
        want = full[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        assert torch.equal(box.view(torch.int64), want.contiguous().view(torch.int64)), (lo, hi)
