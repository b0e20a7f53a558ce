#!/usr/bin/env python
"""STZ B200 benchmark: compress + full decompress of a 512^3 float32 field.

Workload (the reference's headline config): 512x512x512 float32 lognormal field
exp(1.5 g), g a seeded unit-variance Gaussian random field with P(k) ~ k^-3,
value-range-relative error bound 1e-3 (pointwise max|x - x'| <= 1e-3 * range),
zstd level 3 (the reference's final stage). One step = compress (field ->
stream) + full decompress (stream -> field).

  value : field bytes x 2 / step time, field and output resident in HBM, the
          stream in host memory (the zstd stage runs on the host cores).
  e2e   : the same through the host-buffer API: pinned host field in, host
          output back, host<->device copies inside the timed region.

Multi-GPU (torchrun): replicas only — every rank codes its own field, no
collective on the data path; value = all ranks' bytes / max-over-ranks time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sc25-stz2_b200"))

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic.json")
FALLBACK_HBM = 6650.0
METRIC = "compress+decompress GB/s (512^3 f32 lognormal, rel eb 1e-3)"
MULTS = (0.7, 2.7, 8.2)


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--size", type=int, default=512)
    p.add_argument("--rel", type=float, default=1e-3)
    p.add_argument("--zstd", type=int, default=3)
    p.add_argument("--seed", type=int, default=2025)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-parity", action="store_true", help="skip the bit-identity check against oracle/_ref")
    p.add_argument("--once", action="store_true",
                   help="one compress + one full decompress of the workload, no timing (profiler captures)")
    p.add_argument("--no-serve", action="store_true", help="skip the request-server latency measurement")
    p.add_argument("--serve-only", action="store_true", help="only the request-server latency measurement")
    p.add_argument("--serve-trace", default="",
                   help="write per-request (arrival s, queue ms, latency ms, batch, batch size) arrays to this .npz")
    p.add_argument("--serve-size", type=int, default=1024, help="edge of the resident serving field")
    p.add_argument("--serve-seconds", type=float, default=2.0, help="length of each serving load run")
    p.add_argument("--no-learned", action="store_true", help="skip the learned-predictor measurement")
    p.add_argument("--no-configs", action="store_true", help="skip the other BASELINE configurations")
    p.add_argument("--learned-only", action="store_true", help="only the learned-predictor measurement")
    p.add_argument("--learn-train-seeds", type=int, default=6, help="training fields (cycling the 3 generators)")
    p.add_argument("--learn-size", type=int, default=256, help="edge of the training fields")
    p.add_argument("--learn-eval-seeds", type=int, default=3, help="held-out evaluation fields")
    p.add_argument("--learn-eval-size", type=int, default=512, help="edge of the evaluation fields")
    p.add_argument("--learn-full", action="store_true",
                   help="the full protocol: 64 training seeds of 256^3, 8 held-out 512^3 seeds")
    return p.parse_args()


def dist_env():
    from stz_b200.replicas import rank_env

    return rank_env()


# ---- clocks ---------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---- CPU side: the reference's own code, timed on the host cores ------------------
def cpu_reference_round_trip(field: np.ndarray, rel: float, radius: int = 32768) -> dict:
    """One compress+decompress of `field` with the reference's functions
    (oracle/_ref: FD5 split, predict, quantize, closed loop, recover,
    depreprocess, merge) scheduled as FD5 schedules them, OpenMP on all host
    cores. The SZ3-ncp Huffman/zstd stages are not available, so they are not
    included: the CPU does strictly less work than the GPU step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    if not po.ref_available():
        return {}
    R = po.ref()
    suf = "f32" if field.dtype == np.float32 else "f64"
    enc = getattr(R, "fd5ref_level_encode_timed_" + suf)
    enc.restype = C.c_longlong
    enc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
    rec = getattr(R, "fd5ref_recover_parallel_" + suf)
    rec.argtypes = [C.c_void_p, C.c_size_t, C.c_double, C.c_int, C.c_void_p]
    nz, ny, nx = field.shape
    K = po.num_levels(nx, ny, nz)
    rng = float(field.max()) - float(field.min())
    eb = rel * rng / max(MULTS)
    ebk = [0.0] + [(MULTS[2] if k == K else MULTS[1] if k == K - 1 else MULTS[0]) * eb for k in range(1, K + 1)]
    t0 = time.perf_counter()
    coarse = np.ascontiguousarray(field[:: 1 << K, :: 1 << K, :: 1 << K])
    coarsest = coarse
    codes, unpred = [], 0
    for k in range(1, K + 1):
        s = 1 << (K - k)
        fine = field if s == 1 else np.ascontiguousarray(field[::s, ::s, ::s])
        dz, dy, dx = coarse.shape
        q = np.empty(7 * dx * dy * dz, np.int32)
        dec = np.empty(fine.shape, field.dtype) if k < K else None
        unpred += enc(fine.ctypes.data, coarse.ctypes.data, dx, dy, dz, ebk[k], radius, q.ctypes.data,
                      dec.ctypes.data if dec is not None else None)
        codes.append(q)
        coarse = dec
    t1 = time.perf_counter()
    coarse = coarsest
    for k in range(1, K + 1):
        q = codes[k - 1]
        dq = np.empty(q.size, field.dtype)
        rec(q.ctypes.data, q.size, ebk[k], radius, dq.ctypes.data)
        coarse = po.ref_level_decode(dq, coarse, 1 if k == K else 0)
    t2 = time.perf_counter()
    return {"compress_s": t1 - t0, "decompress_s": t2 - t1, "unpred": int(unpred)}


def reference_parity(ctx, stream, field_host: np.ndarray, decoded_host: np.ndarray) -> dict:
    """Bit-identity of the measured stream with the reference's own code
    (oracle/_ref FD5 level functions through the hierarchy, at the eb the
    stream records): every level's quant codes of every block, and the decoded
    field. Runs outside the timed region."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    if not po.ref_available():
        return {"unavailable": "oracle/_ref missing"}
    t0 = time.perf_counter()
    ref = po.ref_round_trip(field_host, stream.info().eb)
    codes_ok = True
    for k in range(1, ref["K"] + 1):
        for b in range(7):
            codes_ok &= bool(np.array_equal(ctx.stream_codes(stream, k, b), ref["codes"][k - 1][b]))
    u = np.uint64 if field_host.dtype == np.float64 else np.uint32
    dec_ok = bool(np.array_equal(decoded_host.view(u), ref["grids"][ref["K"]].view(u)))
    return {"codes": codes_ok, "decoded": dec_ok, "closed_loop": ref["closed_loop_ok"],
            "unpred": int(sum(sum(c) for c in ref["unpred"])),
            "against": "reference FD5 level functions compiled from source (oracle/_ref), same eb",
            "check_s": round(time.perf_counter() - t0, 2)}


def omp_threads(n: int | None) -> None:
    """Set the OpenMP thread count of the reference and oracle libraries
    (they share the process's libgomp); None = all host cores."""
    lib = C.CDLL("libgomp.so.1")
    lib.omp_set_num_threads(int(n if n else cpu_cores()))


def cpu_restated_pipeline(field: np.ndarray, rel: float) -> dict:
    """The whole pipeline on the host cores through the oracle's C
    restatement (levels, codebooks, Huffman, zstd 3, container; the same
    stream as the GPU's): restated, not reference. Its level stages use
    OpenMP, its per-stream entropy stages run one stream at a time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    eb = po.pointwise_eb(field, rel)
    t0 = time.perf_counter()
    b = po.compress(field, eb)
    t1 = time.perf_counter()
    po.decompress(b)
    t2 = time.perf_counter()
    return {"compress_s": t1 - t0, "decompress_s": t2 - t1, "stream_bytes": len(b)}


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def make_field_host(n: int, seed: int) -> np.ndarray:
    import torch
    from stz_b200 import fields

    if torch.cuda.is_available():
        return fields.lognormal((n, n, n), seed, np.float32, device="cuda").cpu().numpy()
    return fields.lognormal((n, n, n), seed, np.float32)


# ---- reference arm ------------------------------------------------------------------
def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    if not po.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libfd5ref.so missing"}))
        return
    n = args.size
    field = make_field_host(n, args.seed)
    sample = field
    # size the sample so the whole run stays within a few minutes
    first = cpu_reference_round_trip(sample, args.rel)
    per = first["compress_s"] + first["decompress_s"]
    while per * (args.steps + args.warmup) > 240 and sample.shape[0] > 64:
        sample = np.ascontiguousarray(sample[: sample.shape[0] // 2])
        r = cpu_reference_round_trip(sample, args.rel)
        per = r["compress_s"] + r["decompress_s"]
    for _ in range(max(0, args.warmup - 1)):
        cpu_reference_round_trip(sample, args.rel)
    times = []
    for _ in range(args.steps):
        r = cpu_reference_round_trip(sample, args.rel)
        times.append(r["compress_s"] + r["decompress_s"])
    total = sum(times)
    gbs = 2 * sample.nbytes * args.steps / total / 1e9
    desc = (f"{sample.shape[2]}x{sample.shape[1]}x{sample.shape[0]} f32 lognormal per step: reference FD5 split/"
            "predict/quantize/closed-loop/recover/depreprocess/merge on all host cores; SZ3-ncp Huffman+zstd "
            "unavailable (not timed)")
    out = {
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic lognormal exp(1.5 g), g GRF k^-3, seed {args.seed}",
        "config": {"workload": "512^3 f32 lognormal, rel eb 1e-3, compress + full decompress",
                   "field": [n, n, n], "rel_eb": args.rel},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": cpu_cores(), "kind": "reference", "sample": desc},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


# ---- serving -------------------------------------------------------------------------
def _pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def serve_load(srv, sid, dims_xyz, K, rate, seconds, gen, seed):
    """Open-loop Poisson load: a producer thread submits at the arrival times,
    a consumer waits for each ticket and releases its output. Latency is the
    server's own submit -> result-complete time."""
    import threading

    rng = np.random.default_rng(seed)
    n = max(1, int(rate * seconds))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = [gen(rng) for _ in range(n)]
    tickets = [0] * n
    ready = threading.Semaphore(0)
    err = []

    def producer():
        t0 = time.perf_counter()
        try:
            for i in range(n):
                while True:
                    dt = arrivals[i] - (time.perf_counter() - t0)
                    if dt <= 0:
                        break
                    time.sleep(min(dt, 2e-4))
                r = reqs[i]
                tickets[i] = srv.submit_box(sid, r[1], r[2]) if r[0] != "level" else srv.submit_level(sid, r[1])
                ready.release()
        except Exception as e:  # reported below
            err.append(repr(e))
            ready.release()

    lat = {"box": [], "slice": [], "level": []}
    batch_sizes, out_bytes, queue, order, trace = [], 0, [], [], []
    th = threading.Thread(target=producer)
    t0 = time.perf_counter()
    th.start()
    for i in range(n):
        ready.acquire()
        if err:
            break
        res = srv.wait(tickets[i])
        srv.release(tickets[i])
        if res.status != 0:
            err.append(f"status {res.status}")
            break
        lat[reqs[i][0]].append(res.latency_ms)
        order.append(res.latency_ms)
        queue.append(res.queue_ms)
        trace.append((arrivals[i], res.queue_ms, res.latency_ms, res.batch, res.batch_size))
        batch_sizes.append(res.batch_size)
        out_bytes += res.nbytes
    wall = time.perf_counter() - t0
    th.join()
    if err:
        return {"error": err[0]}
    allv = [x for v in lat.values() for x in v]
    h = len(order) // 2
    out = {"offered_rps": rate, "requests": n, "achieved_rps": n / wall, "p50_ms": _pct(allv, 50),
           "p99_ms": _pct(allv, 99), "max_ms": max(allv), "queue_p50_ms": _pct(queue, 50),
           "queue_p99_ms": _pct(queue, 99), "p99_first_half_ms": _pct(order[:h], 99),
           "p99_second_half_ms": _pct(order[h:], 99), "mean_batch": float(np.mean(batch_sizes)),
           "max_batch": int(max(batch_sizes)), "out_gbs": out_bytes / wall / 1e9}
    for k, v in lat.items():
        if v:
            out[k] = {"n": len(v), "p50_ms": _pct(v, 50), "p99_ms": _pct(v, 99)}
    out["_trace"] = trace
    return out


def serving_bench(args, ctx, local):
    """Resident-stream request serving on a 1024^3 f32 GRF (P(k) ~ k^-3, rel
    eb 1e-3): 64^3 boxes alone under Poisson load, the mixed workload (60%
    boxes with edges U[16,256], 30% slices, 10% progressive levels 0-3), and
    one-request-at-a-time decode of the same 64^3 boxes through the
    single-request API as the unbatched baseline."""
    import torch

    import stz_b200
    from stz_b200 import fields

    n = args.serve_size
    f = fields.grf((n, n, n), 3.0, args.seed + 1000, np.float32, device=f"cuda:{local}")
    s = ctx.compress(f, opts=stz_b200.default_opts(eb=args.rel, eb_mode="rel", zstd_level=args.zstd))
    E = args.rel * (float(f.max()) - float(f.min()))
    probe = ctx.decompress_box(s, (n // 3, n // 5, n // 7), (n // 3 + 63, n // 5 + 63, n // 7 + 63))
    ref = f[n // 7:n // 7 + 64, n // 5:n // 5 + 64, n // 3:n // 3 + 64].cpu().numpy()
    probe_err = float(np.abs(probe.astype(np.float64) - ref).max()) / E
    del f, ref
    torch.cuda.empty_cache()
    K = s.info().n_levels
    dims = (n, n, n)
    full_bytes = n * n * n * 4
    srv = stz_b200.Server(local, arena_bytes=max(4 << 30, 5 * full_bytes), max_batch=64)
    t0 = time.perf_counter()
    sid = srv.add_stream(s)
    add_s = time.perf_counter() - t0

    def box64(rng):
        lo = [int(rng.integers(0, d - 63)) for d in dims]
        return ("box", lo, [v + 63 for v in lo])

    def mixed(rng):
        u = rng.random()
        if u < 0.6:
            e = [int(rng.integers(16, 257)) for _ in range(3)]
            lo = [int(rng.integers(0, d - x + 1)) for d, x in zip(dims, e)]
            return ("box", lo, [a + x - 1 for a, x in zip(lo, e)])
        if u < 0.9:
            ax = int(rng.integers(0, 3))
            lo, hi = [0, 0, 0], [d - 1 for d in dims]
            lo[ax] = hi[ax] = int(rng.integers(0, dims[ax]))
            return ("slice", lo, hi)
        return ("level", int(rng.integers(0, 4)))

    res = {"field": f"{n}^3 f32 GRF k^-3, rel eb {args.rel}", "stream_bytes": len(s), "cr": full_bytes / len(s),
           "probe_box_max_err_over_bound": probe_err, "add_stream_s": add_s, "shapes": srv.stats()}
    sec = args.serve_seconds
    serve_load(srv, sid, dims, K, 500, 0.2, box64, 1)  # warm-up
    traces = {}
    res["box64"] = []
    box_rates = (2000, 10000, 20000, 50000)
    for i, r in enumerate(box_rates):
        # the top rates run shorter: the Python producer must keep up
        res["box64"].append(serve_load(srv, sid, dims, K, r, sec if r <= 10000 else sec / 2, box64, 10 + i))
        traces[f"box64_{r}_batches"] = srv.batch_log()
    serve_load(srv, sid, dims, K, 200, 0.5, mixed, 2)  # warm-up of the bulk lane (level requests)
    res["mixed"] = serve_load(srv, sid, dims, K, 1000, sec, mixed, 20)
    traces["mixed_batches"] = srv.batch_log()
    for r, b in zip(box_rates, res["box64"]):
        traces[f"box64_{r // 1000}k"] = np.asarray(b.pop("_trace", []), dtype=np.float64)
    traces["mixed"] = np.asarray(res["mixed"].pop("_trace", []), dtype=np.float64)
    if args.serve_trace:
        np.savez(args.serve_trace, **traces)
    srv.close()
    # unbatched baseline: the single-request API on the resident stream
    ctx.upload(s)
    out = torch.empty((64, 64, 64), dtype=torch.float32, device=f"cuda:{local}")
    rng = np.random.default_rng(30)
    lat = []
    for i in range(220):
        r = box64(rng)
        torch.cuda.synchronize()
        t = time.perf_counter()
        ctx.decompress_box(s, r[1], r[2], out=out)
        torch.cuda.synchronize()
        if i >= 20:
            lat.append(1e3 * (time.perf_counter() - t))
    res["box64_one_at_a_time"] = {"requests": len(lat), "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99),
                                  "max_rps": 1e3 / float(np.mean(lat))}
    # the same single-request path under the batched runs' offered loads:
    # Poisson arrivals served one at a time in arrival order (a request waits
    # for the ones before it); latency = completion - arrival
    res["box64_one_at_a_time_under_load"] = []
    for i, rate in enumerate(box_rates):
        rng = np.random.default_rng(10 + i)
        nreq = int(rate * 0.25)
        arr = np.cumsum(rng.exponential(1.0 / rate, nreq))
        reqs = [box64(rng) for _ in range(nreq)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat = []
        for a, r in zip(arr, reqs):
            now = time.perf_counter() - t0
            if now < a:
                time.sleep(a - now)
            ctx.decompress_box(s, r[1], r[2], out=out)
            lat.append(1e3 * (time.perf_counter() - t0 - a))
        res["box64_one_at_a_time_under_load"].append(
            {"offered_rps": rate, "requests": nreq, "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99),
             "achieved_rps": nreq / (time.perf_counter() - t0)})
    return res


def configs_bench(args, ctx, local, field):
    """The other BASELINE configurations, measured (device-resident fields and
    outputs, CUDA events on the library's stream):
    * 512^3 f32 lognormal at rel eb 1e-2 and 1e-4: compress and full
      decompress GB/s, CR;
    * progressive decompress of the rel 1e-3 stream at 1/8, 1/4 and 1/2
      resolution (levels 3, 2, 1): ms and output GB/s;
    * 384x384x256 f64 GRF k^-5/3 + 20 tanh fronts at rel eb 1e-6 and 1e-3:
      100 boxes (edges U[16,128], random offsets) and 20 axis-aligned slices
      through the single-request box API, p50/p99 ms per request, against
      decoding the whole stream and cropping (what a decoder without marker
      chunks must do, the no-marker ROI baseline of src/stz-rd.cpp)."""
    import torch

    import stz_b200
    from stz_b200 import fields

    dev = f"cuda:{local}"
    stream = torch.cuda.ExternalStream(ctx.cuda_stream(), device=dev)
    nbytes = field.numel() * field.element_size()
    out = torch.empty_like(field)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, r

    res = {"eb_sweep": [], "progressive": [], "fronts_384_f64": []}
    for rel in (1e-2, 1e-3, 1e-4):
        o = stz_b200.default_opts(eb=rel, eb_mode="rel", zstd_level=args.zstd)
        cms, s = timed(lambda: ctx.compress(field, opts=o), 3)
        dms, _ = timed(lambda: ctx.decompress(s, out=out), 3)
        res["eb_sweep"].append({"rel_eb": rel, "compress_gbs": nbytes / cms / 1e6, "decompress_gbs": nbytes / dms / 1e6,
                                "cr": nbytes / len(s)})
        if rel == 1e-3:
            for lvl in (3, 2, 1):
                st = 1 << lvl
                o_l = torch.empty((field.shape[0] // st, field.shape[1] // st, field.shape[2] // st),
                                  dtype=field.dtype, device=dev)
                lms, _ = timed(lambda: ctx.decompress(s, level=lvl, out=o_l), 5)
                res["progressive"].append({"level": lvl, "resolution": f"1/{st}", "ms": lms,
                                           "output_gbs": o_l.numel() * 4 / lms / 1e6,
                                           "field_equiv_gbs": nbytes / lms / 1e6})
    # predictor modes on the same field and bound, at the multipliers of the
    # reference's artifact programs (1 / 2.5 / 6.25, float.cpp and
    # dependency.cpp): the staged predictor of src/dependency.cpp against the
    # dynamic lines (FD5) and the plain cubic stencils (float.cpp), and the
    # 12-point truncated bicubic of src/stz2.cpp
    res["predictors"] = []
    for name in ("dynamic", "cubic", "staged", "truncated"):
        try:
            o = stz_b200.default_opts(eb=1e-3, eb_mode="rel", zstd_level=args.zstd, predictor=name, mult_base=1.0,
                                      mult_low=2.5, mult_high=6.25)
            cms, s = timed(lambda: ctx.compress(field, opts=o), 3)
            dms, _ = timed(lambda: ctx.decompress(s, out=out), 3)
            res["predictors"].append({"predictor": name, "rel_eb": 1e-3, "mults": [1.0, 2.5, 6.25],
                                      "compress_gbs": nbytes / cms / 1e6, "decompress_gbs": nbytes / dms / 1e6,
                                      "cr": nbytes / len(s)})
            del s
        except Exception as e:  # recorded, so the rest of the line still comes out
            res["predictors"].append({"predictor": name, "error": str(e)[:200]})
    del out
    torch.cuda.empty_cache()
    nz, ny, nx = 256, 384, 384
    f = fields.fronts((nz, ny, nx), 31, np.float64, device=dev)
    dims = (nx, ny, nz)
    for rel in (1e-6, 1e-3):
        s = ctx.compress(f, eb=rel, eb_mode="rel")
        ctx.upload(s)
        rng = np.random.default_rng(int(1 / rel) % 1000)
        reqs = []
        for _ in range(100):
            e = rng.integers(16, 129, 3)
            lo = [int(rng.integers(0, d - x + 1)) for d, x in zip(dims, e)]
            reqs.append(("box", lo, [a + int(x) - 1 for a, x in zip(lo, e)]))
        for _ in range(20):
            ax = int(rng.integers(0, 3))
            lo, hi = [0, 0, 0], [d - 1 for d in dims]
            lo[ax] = hi[ax] = int(rng.integers(0, dims[ax]))
            reqs.append(("slice", lo, hi))
        lat = {"box": [], "slice": []}
        for kind, lo, hi in reqs[:5]:  # warm-up
            ctx.decompress_box(s, lo, hi, out=torch.empty((hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1),
                                                          dtype=f.dtype, device=dev))
        for kind, lo, hi in reqs:
            o_b = torch.empty((hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1), dtype=f.dtype, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.decompress_box(s, lo, hi, out=o_b)
            torch.cuda.synchronize()
            lat[kind].append(1e3 * (time.perf_counter() - t0))
        full = torch.empty_like(f)
        whole = []
        for kind, lo, hi in reqs[:20]:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.decompress(s, out=full)
            crop = full[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1].contiguous()
            torch.cuda.synchronize()
            whole.append(1e3 * (time.perf_counter() - t0))
        del full, crop
        res["fronts_384_f64"].append({
            "rel_eb": rel, "cr": f.numel() * 8 / len(s),
            "box_p50_ms": _pct(lat["box"], 50), "box_p99_ms": _pct(lat["box"], 99),
            "slice_p50_ms": _pct(lat["slice"], 50), "slice_p99_ms": _pct(lat["slice"], 99),
            "whole_stream_then_crop_p50_ms": _pct(whole, 50)})
    del f
    torch.cuda.empty_cache()
    return res


def learned_bench(args, ctx, local, field):
    """Learned correction: train on seeded 256^3 f32 fields cycling the three
    generators (GRF k^-11/3, lognormal, GRF k^-5/3 + fronts) at rel eb 1e-3
    with the library's GPU trainer; on held-out 512^3 seeds at rel eb 1e-3 and
    1e-4 compare stream size (CR) and PSNR with and without the model (the
    per-block flags choose); time compress + decompress of the benchmark field
    with the learned kernels forced on every block of both levels."""
    import torch

    import stz_b200
    from stz_b200 import fields

    dev = f"cuda:{local}"
    gens = ("grf", "logn", "fronts")

    def gen_field(g, e, seed):
        shape = (e, e, e)
        if g == "grf":
            return fields.grf(shape, 11.0 / 3.0, seed, np.float32, device=dev)
        if g == "logn":
            return fields.lognormal(shape, seed, np.float32, device=dev)
        return fields.fronts(shape, seed, np.float32, device=dev)

    ntrain = 64 if args.learn_full else args.learn_train_seeds
    neval = 8 if args.learn_full else args.learn_eval_seeds
    topts = stz_b200.default_train_opts()
    tr = stz_b200.Trainer(ctx, train=topts, eb=1e-3, eb_mode="rel", zstd_level=args.zstd)
    t0 = time.perf_counter()
    for i in range(ntrain):
        f = gen_field(gens[i % 3], args.learn_size, 5000 + i)
        tr.add_field(f)
        del f
    torch.cuda.synchronize()
    pairs_s = time.perf_counter() - t0
    model = tr.fit()
    st = tr.stats()
    tr.close()
    rows = []
    for j in range(neval):
        g = gens[j % 3]
        f = gen_field(g, args.learn_eval_size, 9000 + j)
        vr = float(f.max()) - float(f.min())
        out = torch.empty_like(f)
        for rel in (1e-3, 1e-4):
            row = {"generator": g, "seed": 9000 + j, "rel_eb": rel}
            for name, kw in (("plain", {}), ("learned", {"model": model})):
                s = ctx.compress(f, eb=rel, eb_mode="rel", zstd_level=args.zstd, **kw)
                ctx.decompress(s, out=out)
                mse = float(((out.double() - f.double()) ** 2).mean())
                row[name] = {"bytes": len(s), "cr": f.numel() * 4 / len(s),
                             "psnr_db": 20 * np.log10(vr) - 10 * np.log10(max(mse, 1e-300)),
                             "max_err_over_bound": float((out.double() - f.double()).abs().max()) / (rel * vr)}
                if name == "learned":
                    row["learned_flags"] = s.info().learned_flags
            row["cr_gain"] = row["learned"]["cr"] / row["plain"]["cr"]
            rows.append(row)
        del f, out
    torch.cuda.empty_cache()
    # throughput with every block of both levels corrected
    out = torch.empty_like(field)
    stream = torch.cuda.ExternalStream(ctx.cuda_stream(), device=dev)
    thr = {}
    all_blocks = {"model": model, "learned_flags": 0x7F7F}
    ref_bytes = None
    for name, kw, path in (("plain", {}, "tc"), ("learned_all_blocks", all_blocks, "tc"),
                           ("learned_all_blocks_dp4a", all_blocks, "dp4a")):
        os.environ["STZ_LEARNED_PATH"] = path
        o = stz_b200.default_opts(eb=args.rel, eb_mode="rel", zstd_level=args.zstd, **kw)
        for _ in range(2):
            s = ctx.compress(field, opts=o)
            ctx.decompress(s, out=out)
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        steps = max(2, args.steps)
        cms = dms = 0.0
        ctx.profile(True)
        ctx.profile_reset()
        for _ in range(steps):
            e[0].record(stream)
            s = ctx.compress(field, opts=o)
            e[1].record(stream)
            ctx.decompress(s, out=out)
            e[2].record(stream)
            torch.cuda.synchronize()
            cms += e[0].elapsed_time(e[1])
            dms += e[1].elapsed_time(e[2])
        prof = ctx.profile_read()
        ctx.profile(False)
        nb = field.numel() * 4
        thr[name] = {"compress_gbs": nb * steps / cms / 1e6, "decompress_gbs": nb * steps / dms / 1e6,
                     "cr": nb / len(s), "level_kernel_ms": {k: round(v[0] / steps, 4) for k, v in prof.items()
                                                            if k.startswith("k_level")}}
        if kw:  # both learned paths write the same stream
            b = s.to_bytes()
            thr[name]["same_stream_as_other_path"] = None if ref_bytes is None else b == ref_bytes
            ref_bytes = b
    os.environ.pop("STZ_LEARNED_PATH", None)
    del out
    gains = {}
    for rel in (1e-3, 1e-4):
        v = [r["cr_gain"] for r in rows if r["rel_eb"] == rel]
        gains[str(rel)] = float(np.exp(np.mean(np.log(v)))) if v else None
    return {"train": {"fields": ntrain, "edge": args.learn_size, "rel_eb": 1e-3, "pairs": st["pairs"],
                      "pair_extraction_s": pairs_s, "fit_ms": st["train_ms"],
                      "loss_zero": st["loss_zero"], "loss_float": st["loss_float"], "loss_qat": st["loss_qat"],
                      "loss_int8": st["loss_int8"],
                      "opts": {"epochs": topts.epochs, "qat_epochs": topts.qat_epochs, "batch": topts.batch,
                               "lr": topts.lr, "huber_delta": topts.huber_delta, "sample_step": topts.sample_step}},
            "eval": rows, "cr_gain_geomean": gains, "throughput": thr,
            "throughput_ratio_learned_vs_plain": {
                "compress": thr["learned_all_blocks"]["compress_gbs"] / thr["plain"]["compress_gbs"],
                "decompress": thr["learned_all_blocks"]["decompress_gbs"] / thr["plain"]["decompress_gbs"],
                "compress_dp4a": thr["learned_all_blocks_dp4a"]["compress_gbs"] / thr["plain"]["compress_gbs"],
                "decompress_dp4a": thr["learned_all_blocks_dp4a"]["decompress_gbs"] / thr["plain"]["decompress_gbs"]}}


# ---- our arm ---------------------------------------------------------------------------
def algorithmic_bytes(kernel: str, N: int, elem: int, K: int, raw_payload: int) -> float | None:
    """Minimum HBM bytes all launches of `kernel` in one step must move on the N-point field."""
    fine_syms = 7 * N // 8
    all_syms = sum(7 * (N >> (3 * j)) // 8 for j in range(K))
    if kernel == "k_level_encode[finest]":
        return fine_syms * elem + (N // 8) * elem + fine_syms * 2  # read 7 parities + ref grid, write codes
    if kernel == "k_level_decode[finest]":
        return fine_syms * 2 + (N // 8) * elem + N * elem  # read codes + ref grid, write the full field
    if kernel == "k_decode":
        return raw_payload + all_syms * 2  # read payload, write codes
    if kernel == "k_encode":
        return all_syms * 2 + raw_payload  # read codes, write payload
    if kernel == "k_sub_bits" or kernel == "k_run_stats":
        return all_syms * 2
    if kernel == "k_minmax":
        return N * elem
    return None


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    import stz_b200
    from stz_b200 import fields, replicas

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=120, device=torch.device("cuda", local))
    n = args.size
    ctx = stz_b200.Context(local)
    field = fields.lognormal((n, n, n), replicas.replica_seed(args.seed, rank), np.float32, device=f"cuda:{local}")
    nbytes = field.numel() * field.element_size()
    out = torch.empty_like(field)
    opts = stz_b200.default_opts(eb=args.rel, eb_mode="rel", zstd_level=args.zstd)
    stream = torch.cuda.ExternalStream(ctx.cuda_stream(), device=f"cuda:{local}")
    if args.serve_only:
        if rank == 0:
            print(json.dumps({"serving": serving_bench(args, ctx, local)}))
        ctx.close()
        replicas.finalize()
        return
    if args.learned_only:
        if rank == 0:
            print(json.dumps({"learned": learned_bench(args, ctx, local, field)}))
        ctx.close()
        replicas.finalize()
        return
    if args.once:
        s = ctx.compress(field, opts=opts)
        ctx.decompress(s, out=out)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"once": True, "field": [n, n, n], "stream_bytes": len(s)}))
        ctx.close()
        replicas.finalize()
        return

    def step():
        s = ctx.compress(field, opts=opts)
        ctx.decompress(s, out=out)
        return s

    for _ in range(args.warmup):
        s = step()
    torch.cuda.synchronize()
    # correctness of the measured configuration
    E = args.rel * (float(field.max()) - float(field.min()))
    max_err = float((out.double() - field.double()).abs().max())
    cr = nbytes / len(s)
    info = s.info()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    replicas.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    ev[0].record(stream)
    for i in range(args.steps):
        s = ctx.compress(field, opts=opts)
        ev[2 * i + 1].record(stream)
        ctx.decompress(s, out=out)
        ev[2 * i + 2].record(stream)
    torch.cuda.synchronize()
    # per-kernel times: the same K steps once more with the library's
    # per-launch CUDA events (two event records per kernel would add their
    # host cost to the step time above)
    ctx.profile(True)
    ctx.profile_reset()
    for i in range(args.steps):
        s = ctx.compress(field, opts=opts)
        ctx.decompress(s, out=out)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    replicas.barrier()
    clk = clocks.stop()
    comp_ms = sum(ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(args.steps))
    dec_ms = sum(ev[2 * i + 1].elapsed_time(ev[2 * i + 2]) for i in range(args.steps))
    total_ms = replicas.max_over_ranks(ev[0].elapsed_time(ev[-1]), device="cuda")
    comp_ms = replicas.max_over_ranks(comp_ms, device="cuda")
    dec_ms = replicas.max_over_ranks(dec_ms, device="cuda")
    value = replicas.aggregate_gbs(2 * nbytes * args.steps, world, total_ms)
    launches = int(sum(v[1] for v in prof.values()))

    # end to end through the host-buffer API
    e2e = None
    if not args.no_e2e:
        host_field = field.cpu().pin_memory()
        host_out_t = torch.empty((n, n, n), dtype=torch.float32, pin_memory=True)
        host_out = host_out_t.numpy()
        s = ctx.compress(host_field, opts=opts)
        ctx.decompress(s, out=host_out)
        replicas.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            s = ctx.compress(host_field, opts=opts)
            ctx.decompress(s, out=host_out)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda")
        inf = s.info()
        assert np.array_equal(host_out.view(np.uint32), out.cpu().numpy().view(np.uint32))
        # the link itself: pinned copies of the field each way, same buffers
        dev_tmp = torch.empty_like(field)
        torch.cuda.synchronize()
        l0, l1, l2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        l0.record()
        for _ in range(3):
            dev_tmp.copy_(host_field, non_blocking=True)
        l1.record()
        for _ in range(3):
            host_out_t.copy_(dev_tmp, non_blocking=True)
        l2.record()
        torch.cuda.synchronize()
        h2d = 3 * nbytes / (l0.elapsed_time(l1) / 1e3) / 1e9
        d2h = 3 * nbytes / (l1.elapsed_time(l2) / 1e3) / 1e9
        del dev_tmp
        # both transfers of a step back to back, no compute: the most e2e can be
        link_bound = 2 * nbytes / (nbytes / (h2d * 1e9) + nbytes / (d2h * 1e9)) / 1e9
        e2e_v = replicas.aggregate_gbs(2 * nbytes * args.steps, world, e2e_ms)
        e2e = {"value": e2e_v, "unit": "GB/s",
               "h2d_bytes_per_step": nbytes + inf.raw_payload_bytes,
               "d2h_bytes_per_step": nbytes + inf.raw_payload_bytes,
               "host_buffers": "pinned field in, pinned output back",
               "link_h2d_gbs": h2d, "link_d2h_gbs": d2h, "link_bound_gbs": link_bound,
               "frac_of_link_bound": e2e_v / world / link_bound}

    # roofline of the dominant kernel
    peaks = {}
    if os.path.exists(PEAKS_FILE):
        peaks = json.load(open(PEAKS_FILE))
    peak = peaks.get("hbm_gbs", FALLBACK_HBM)
    traffic_tab = json.load(open(TRAFFIC_FILE)) if os.path.exists(TRAFFIC_FILE) else {}

    def roofline_of(name):
        dms, dl = prof[name]
        alg = algorithmic_bytes(name, field.numel(), 4, info.n_levels, info.raw_payload_bytes)
        if alg is None or not dl:
            return None
        # alg covers one step; a kernel launched several times per step (the
        # coder's stream batches, the finest decode's z-halves) moves
        # alg / (launches per step) per launch
        alg = alg * args.steps / dl
        per_launch_s = dms / dl / 1e3
        achieved = alg / per_launch_s / 1e9
        tr = traffic_tab.get(name) or {}
        return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": tr.get("dram_bytes_per_launch"), "algorithmic_bytes": alg,
                "ms_per_launch": dms / dl, "launches_per_step": dl / args.steps,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "timing": "per-launch CUDA events on the launching stream, over a second pass of the K timed steps"}

    # the dominant kernel (most time per step) and every kernel with a
    # roofline, so a change of the top kernel does not hide the others
    dname = max(prof.items(), key=lambda kv: kv[1][0])[0]
    roof = roofline_of(dname)
    rooflines = {k: r for k in prof for r in [roofline_of(k)] if r}

    parity = None
    if rank == 0 and not args.no_parity:
        parity = reference_parity(ctx, s, field.cpu().numpy(), out.cpu().numpy())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fh = field.cpu().numpy()
        r = cpu_reference_round_trip(fh, args.rel)
        if r:
            sec = r["compress_s"] + r["decompress_s"]
            cpu = {"value": 2 * nbytes / sec / 1e9, "unit": "GB/s", "cores": cpu_cores(), "kind": "reference",
                   "sample": f"one full {n}^3 round trip: reference FD5 split/predict/quantize/closed-loop/recover/"
                             "depreprocess/merge, OpenMP on all host cores; SZ3-ncp Huffman+zstd unavailable "
                             "(not timed)",
                   "compress_s": r["compress_s"], "decompress_s": r["decompress_s"]}
            # the same reference stages on one core (a 128-plane slab of the field, scaled)
            omp_threads(1)
            slab = np.ascontiguousarray(fh[:128])
            r1 = cpu_reference_round_trip(slab, args.rel)
            omp_threads(None)
            s1 = r1["compress_s"] + r1["decompress_s"]
            cpu["serial"] = {"value": 2 * slab.nbytes / s1 / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
                             "sample": f"{n}x{n}x128 slab of the field, same reference stages, OMP_NUM_THREADS=1"}
            rp = cpu_restated_pipeline(fh, args.rel)
            sp = rp["compress_s"] + rp["decompress_s"]
            cpu["restated_pipeline"] = {
                "value": 2 * nbytes / sp / 1e9, "unit": "GB/s", "cores": cpu_cores(), "kind": "restated, not reference",
                "sample": f"one full {n}^3 round trip through the C restatement (oracle/): levels, codebooks, "
                          "Huffman, zstd 3, container, the GPU's stream byte for byte",
                "compress_s": rp["compress_s"], "decompress_s": rp["decompress_s"]}

    cfgs = None
    if rank == 0 and world == 1 and not args.no_configs:
        cfgs = configs_bench(args, ctx, local, field)

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        serving = serving_bench(args, ctx, local)
    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        learned = learned_bench(args, ctx, local, field)

    if rank == 0:
        head = {}
        if serving and "box64" in serving:
            for b in serving["box64"]:
                if "p99_ms" in b:
                    head[f"box64_p99_ms_at_{int(b['offered_rps']) // 1000}k"] = round(b["p99_ms"], 3)
                    head[f"box64_mean_batch_at_{int(b['offered_rps']) // 1000}k"] = round(b["mean_batch"], 2)
            mx = serving.get("mixed", {})
            if "box" in mx:
                head["mixed_box_p99_ms"] = round(mx["box"]["p99_ms"], 3)
        if learned:
            head["learned_cr_gain_geomean"] = learned.get("cr_gain_geomean")
        if parity:
            head["parity_codes"], head["parity_decoded"] = parity.get("codes"), parity.get("decoded")
        res = {
            "metric": METRIC, "value": value, "unit": "GB/s", "headline": head, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": f"synthetic lognormal exp(1.5 g), g GRF k^-3 (FFT-filtered seeded white noise), seed {args.seed}+rank",
            "config": {"workload": "512^3 f32 lognormal, rel eb 1e-3, compress + full decompress",
                       "field": [n, n, n], "rel_eb": args.rel, "zstd_level": args.zstd,
                       "l2": "inputs larger than L2 (512 MiB field per step)", "parallelism": f"replicas x{world}"},
            "compress_gbs": replicas.aggregate_gbs(nbytes * args.steps, world, comp_ms),
            "decompress_gbs": replicas.aggregate_gbs(nbytes * args.steps, world, dec_ms),
            "parity": parity, "cr": cr, "max_err_over_bound": max_err / E, "stream_bytes": len(s),
            "e2e": e2e, "gpu_launches": launches, "roofline": roof,
            "rooflines": {k: {kk: r[kk] for kk in ("frac", "achieved", "ms_per_launch", "launches_per_step", "traffic")}
                          for k, r in rooflines.items()},
            "cpu_baseline": cpu, "clocks": clk,
            "configs": cfgs, "serving": serving, "learned": learned,
            "kernel_ms": {k: round(v[0] / args.steps, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
        }
        print(json.dumps(res))
    ctx.close()
    replicas.finalize()


if __name__ == "__main__":
    main()
