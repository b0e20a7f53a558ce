"""The allocation-free quantizer entry point, stz_quantize_noalloc_dev.

Callers that cannot allocate device memory (code inside another framework's
memory pool, latency-critical loops that must not hit the implicit device
synchronization of cudaMalloc/cudaFree, hosts that reserve all GPU memory up
front) use this entry point instead of stz_quantize_dev. It keeps its scratch
in a fixed array inside the library, so its results must equal the regular
entry point's on every call, including a call that follows another one and
finds the previous call's leftovers in that shared scratch.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

import stz_b200

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _data(n, dtype, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(n) * rng.choice([1e-3, 1.0, 1e4], n)
    d[:4] = [0.0, -0.0, np.inf, np.nan]  # unpredictable on purpose
    return torch.from_numpy(d.astype(dtype)).cuda()


def _regular(ctx, d, eb, radius):
    q = torch.zeros(d.numel(), dtype=torch.int32, device="cuda")
    u = torch.zeros_like(d)
    n = ctx.quantize(d, eb, radius, q, u)
    return q.cpu().numpy(), u[:n].cpu().numpy()


def _noalloc(d, eb, radius, stream=None):
    """Run the entry point on `stream` (a torch.cuda.Stream; None = the legacy
    default stream). The outputs are filled on torch's current stream first,
    so the caller's stream waits for that work before the call."""
    q = torch.full((d.numel(),), -7, dtype=torch.int32, device="cuda")
    u = torch.zeros_like(d)
    handle = 0
    if stream is not None:
        stream.wait_stream(torch.cuda.current_stream())
        handle = stream.cuda_stream
    else:
        torch.cuda.current_stream().synchronize()
    n = stz_b200.quantize_noalloc(d, eb, radius, q, u, handle)
    return q.cpu().numpy(), u[:n].cpu().numpy()


def test_noalloc_quantize_matches_regular_entry_point_twice_in_a_row():
    with stz_b200.Context(0) as ctx:
        # first call: large input (many tiles of scratch)
        a = _data(1_000_003, np.float32, 1)
        want_q, want_u = _regular(ctx, a, 1e-2, 32768)
        got_q, got_u = _noalloc(a, 1e-2, 32768)
        assert np.array_equal(got_q, want_q)
        assert got_u.size == want_u.size > 0
        assert np.array_equal(got_u.view(np.uint32), want_u.view(np.uint32))
        # second call right after: smaller, other dtype and bound, on a
        # caller-owned stream; the scratch still holds the first call's data
        b = _data(300_001, np.float64, 2)
        want_q, want_u = _regular(ctx, b, 3e-4, 512)
        s = torch.cuda.Stream()
        got_q, got_u = _noalloc(b, 3e-4, 512, s)
        assert np.array_equal(got_q, want_q)
        assert got_u.size == want_u.size > 0
        assert np.array_equal(got_u.view(np.uint64), want_u.view(np.uint64))


def test_noalloc_quantize_at_its_size_limit():
    """Exactly STZ_NOALLOC_MAX_VALUES values: every tile slot of the fixed
    scratch is used; twice in a row, on a caller-owned stream."""
    n = stz_b200.NOALLOC_MAX_VALUES
    with stz_b200.Context(0) as ctx:
        d = _data(n, np.float32, 3)
        want_q, want_u = _regular(ctx, d, 1e-2, 32768)
        s = torch.cuda.Stream()
        for _ in range(2):
            got_q, got_u = _noalloc(d, 1e-2, 32768, s)
            assert np.array_equal(got_q, want_q)
            assert got_u.size == want_u.size > 0
            assert np.array_equal(got_u.view(np.uint32), want_u.view(np.uint32))


def test_noalloc_quantize_rejects_sizes_beyond_its_scratch():
    lib = stz_b200.load_library()
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    q = torch.zeros(16, dtype=torch.int32, device="cuda")
    n = C.c_size_t(123)
    st = lib.stz_quantize_noalloc_dev(0, C.c_void_p(d.data_ptr()), stz_b200.NOALLOC_MAX_VALUES + 1, 1e-3, 32768,
                                      C.c_void_p(q.data_ptr()), C.c_void_p(d.data_ptr()), C.byref(n), None)
    assert st == 7  # STZ_ERR_RANGE, before any GPU work
    assert b"at most" in lib.stz_last_error()
