"""Request server (stz_server_*): every result equals the single-request
decode (itself pinned to the oracle) whether a request runs alone or inside a
batch, under concurrent submitters, and under output-memory admission."""
import threading

import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def bits(a):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def make_field(gen, shape, dtype, seed):
    from stz_b200 import fields

    if gen == "grf":
        return fields.grf(shape, 11.0 / 3.0, seed, dtype)
    if gen == "logn":
        return fields.lognormal(shape, seed, dtype)
    return fields.fronts(shape, seed, dtype)


def random_requests(rng, dims_xyz, n, levels):
    """Boxes with uneven edges, slices on random axes, progressive levels."""
    reqs = []
    for i in range(n):
        kind = rng.random()
        if kind < 0.6:
            e = [int(rng.integers(1, max(2, d // 2))) for d in dims_xyz]
            lo = [int(rng.integers(0, d - ei + 1)) for d, ei in zip(dims_xyz, e)]
            hi = [l + ei - 1 for l, ei in zip(lo, e)]
            reqs.append(("box", lo, hi))
        elif kind < 0.9:
            ax = int(rng.integers(0, 3))
            lo = [0, 0, 0]
            hi = [d - 1 for d in dims_xyz]
            v = int(rng.integers(0, dims_xyz[ax]))
            lo[ax] = hi[ax] = v
            reqs.append(("box", lo, hi))
        else:
            reqs.append(("level", int(rng.choice(levels))))
    return reqs


def submit(srv, sid, r):
    if r[0] == "box":
        return srv.submit_box(sid, r[1], r[2])
    return srv.submit_level(sid, r[1])


def expected(ctx, s, r):
    if r[0] == "box":
        return ctx.decompress_box(s, r[1], r[2])
    return ctx.decompress(s, level=r[1])


@pytest.fixture(scope="module")
def server():
    from stz_b200 import Server

    srv = Server(0, arena_bytes=256 << 20, max_batch=32)
    yield srv
    srv.close()


@pytest.mark.parametrize("case", [("grf", (64, 64, 128), np.float32, 1e-3, 16, 8),
                                  ("fronts", (64, 64, 64), np.float64, 1e-6, 16, 8)])
def test_results_equal_single_decode_alone_and_in_mix(ctx, server, case):
    gen, shape, dtype, eb, ch, cl = case
    f = make_field(gen, shape, dtype, 11)
    s = ctx.compress(f, eb=eb, eb_mode="rel", chunk_high=ch, chunk_low=cl)
    sid = server.add_stream(s)
    K = s.info().n_levels
    rng = np.random.default_rng(5)
    reqs = random_requests(rng, (shape[2], shape[1], shape[0]), 40, list(range(K + 1)))
    want = [expected(ctx, s, r) for r in reqs]
    # alone: one request in flight at a time
    alone = []
    for r in reqs:
        t = submit(server, sid, r)
        res = server.wait(t)
        assert res.status == 0 and res.batch_size == 1
        alone.append(server.copy_out(res, dtype))
        server.release(t)
    # mixed: everything submitted at once, batched by the server
    tickets = [submit(server, sid, r) for r in reqs]
    results = [server.wait(t) for t in tickets]
    assert max(r.batch_size for r in results) > 1
    mixed = [server.copy_out(r, dtype) for r in results]
    for t in tickets:
        server.release(t)
    for r, w, a, m in zip(reqs, want, alone, mixed):
        assert a.shape == w.shape and m.shape == w.shape, r
        assert np.array_equal(bits(a), bits(w)), r
        assert np.array_equal(bits(m), bits(w)), r
    # a few against the oracle directly
    b = s.to_bytes()
    for r, m in list(zip(reqs, mixed))[:6]:
        if r[0] == "box":
            assert np.array_equal(bits(m), bits(po.decompress_box(b, r[1], r[2]))), r
        else:
            assert np.array_equal(bits(m), bits(po.decompress(b, r[1]))), r
    st = server.stats()
    assert st["completed"] == st["submitted"] and st["arena_in_use"] == 0


def test_concurrent_submitters_and_two_streams(ctx):
    from stz_b200 import Server

    f1 = make_field("grf", (64, 64, 64), np.float32, 21)
    f2 = make_field("logn", (32, 64, 128), np.float32, 22)
    s1 = ctx.compress(f1, eb=1e-3, eb_mode="rel", chunk_high=16, chunk_low=8)
    s2 = ctx.compress(f2, eb=1e-3, eb_mode="rel", chunk_high=16, chunk_low=8)
    full1, full2 = ctx.decompress(s1), ctx.decompress(s2)
    with Server(0, arena_bytes=64 << 20, max_batch=16) as srv:
        ids = [srv.add_stream(s1), srv.add_stream(s2)]
        fulls = [full1, full2]
        dims = [(64, 64, 64), (128, 64, 32)]
        errors = []

        def client(k):
            rng = np.random.default_rng(100 + k)
            try:
                for _ in range(25):
                    j = int(rng.integers(0, 2))
                    d = dims[j]
                    lo = [int(rng.integers(0, x)) for x in d]
                    hi = [min(x - 1, l + int(rng.integers(0, 40))) for x, l in zip(d, lo)]
                    t = srv.submit_box(ids[j], lo, hi)
                    res = srv.wait(t)
                    got = srv.copy_out(res, np.float32)
                    srv.release(t)
                    want = fulls[j][lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
                    if not np.array_equal(bits(got), bits(want)):
                        errors.append((k, j, lo, hi))
            except Exception as e:  # surfaced below
                errors.append(repr(e))

        th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errors, errors[:3]
        st = srv.stats()
        assert st["completed"] == st["submitted"] == 100


def test_admission_by_output_memory(ctx):
    from stz_b200 import Server, StzError

    f = make_field("grf", (64, 64, 64), np.float32, 31)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel", chunk_high=16, chunk_low=8)
    full = ctx.decompress(s)
    box_bytes = 32 * 32 * 32 * 4
    with Server(0, arena_bytes=3 * box_bytes, max_batch=8, autotune=False) as srv:
        sid = srv.add_stream(s)
        with pytest.raises(StzError):
            srv.submit_level(sid, 0)  # 1 MiB output never fits a 384 KiB arena
        corners = [(x, y, z) for x in (0, 32) for y in (0, 32) for z in (0, 32)]
        tickets = [srv.submit_box(sid, c, [v + 31 for v in c]) for c in corners]
        # at most three outputs fit at once: the rest wait for releases
        for c, t in zip(corners, tickets):
            res = srv.wait(t, timeout_ms=20000)
            assert res.status == 0
            assert srv.stats()["arena_in_use"] <= 3 * box_bytes
            got = srv.copy_out(res, np.float32)
            x, y, z = c
            assert np.array_equal(bits(got), bits(full[z:z + 32, y:y + 32, x:x + 32]))
            srv.release(t)
        assert srv.stats()["arena_in_use"] == 0


def test_fast_lane_reserve_admits_boxes_while_full_decodes_hold_memory(ctx):
    """Full decodes (bulk lane) may not take the fast-lane reserve: with the
    rest of the arena held by unreleased full decodes, a box is still served."""
    from stz_b200 import Server, StzError

    f = make_field("grf", (32, 32, 32), np.float32, 43)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel", chunk_high=8, chunk_low=4)
    full = ctx.decompress(s)
    with Server(0, arena_bytes=1 << 20, autotune=False, fast_reserve=256 << 10) as srv:
        sid = srv.add_stream(s)
        held = [srv.submit_level(sid, 0) for _ in range(6)]  # 6 x 128 KiB = the non-reserved 768 KiB
        for t in held:
            assert srv.wait(t, timeout_ms=20000).status == 0
        extra = srv.submit_level(sid, 0)
        with pytest.raises(StzError):
            srv.wait(extra, timeout_ms=200)  # the reserve is not for full decodes
        box = srv.submit_box(sid, (0, 0, 0), (31, 31, 31))  # 128 KiB from the reserve
        res = srv.wait(box, timeout_ms=20000)
        assert np.array_equal(bits(srv.copy_out(res, np.float32)), bits(full))
        srv.release(box)
        srv.release(held[0])
        assert srv.wait(extra, timeout_ms=20000).status == 0
        for t in held[1:] + [extra]:
            srv.release(t)
    # a full decode larger than the arena less the reserve is refused at submit
    with Server(0, arena_bytes=1 << 20, autotune=False, fast_reserve=(1 << 20) - 4096) as srv2:
        sid2 = srv2.add_stream(s)
        with pytest.raises(StzError):
            srv2.submit_level(sid2, 0)
        t = srv2.submit_box(sid2, (0, 0, 0), (31, 31, 31))
        assert srv2.wait(t, timeout_ms=20000).status == 0
        srv2.release(t)


def test_wait_times_out_and_bad_requests(ctx):
    from stz_b200 import Server, StzError

    f = make_field("grf", (32, 32, 32), np.float32, 41)
    s = ctx.compress(f, eb=1e-3, eb_mode="rel", chunk_high=8, chunk_low=4)
    with Server(0, arena_bytes=1 << 20, autotune=False, fast_reserve=0) as srv:
        sid = srv.add_stream(s)
        with pytest.raises(StzError):
            srv.submit_level(sid, 99)
        with pytest.raises(StzError):
            srv.submit_box(sid + 5, (0, 0, 0), (1, 1, 1))
        # fill the 1 MiB arena with eight 128 KiB full decodes: the ninth
        # request waits in the queue until one of them is released
        blockers = [srv.submit_level(sid, 0) for _ in range(8)]
        for t in blockers:
            assert srv.wait(t, timeout_ms=20000).status == 0
        late = srv.submit_level(sid, 0)
        with pytest.raises(StzError):
            srv.wait(late, timeout_ms=200)
        srv.release(blockers[3])
        assert srv.wait(late, timeout_ms=20000).status == 0
        for t in blockers[:3] + blockers[4:] + [late]:
            srv.release(t)
        assert srv.stats()["arena_in_use"] == 0
