"""Generate tests/golden/fd5_golden.npz from the reference's own code.

Runs the reference FD5 functions (oracle/_ref/libfd5ref.so, compiled from the
reference sources by oracle/Makefile) over the hierarchy this project uses:
every refinement level is one call of the reference's level step (slice,
preprocess_block_zslab, quantize_range_nodec and, on coarser levels, the
writeDec closed loop with depreprocess_block_zslab + merge), and the field is
rebuilt with the reference decoder (recover LUT + depreprocess_block_zslab /
depreprocess_block_zslab_to_full). Also records reference planner output for
random queries, the plain tricubic stencils of src/stz-rd.cpp, a staged
pipeline of src/dependency.cpp's stage functions (oracle/_ref/libdep_ref.so)
and the pipeline of src/stz2.cpp's functions (oracle/_ref/libstz2_ref.so).

    python tests/golden/make_golden.py        # needs the reference sources
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "sc25-stz2_b200"))

import pyoracle as po  # noqa: E402
from stz_b200 import fields  # noqa: E402

MULTS = (0.7, 2.7, 8.2)
RADIUS = 32768


def hierarchy(field: np.ndarray, rel: float):
    nz, ny, nx = field.shape
    K = po.num_levels(nx, ny, nz)
    eb = po.pointwise_eb(field, rel, MULTS)
    out = {"eb": np.float64(eb), "K": np.int64(K)}
    G = np.ascontiguousarray(field[:: 1 << K, :: 1 << K, :: 1 << K])
    out["coarsest"] = G.copy()
    coarse = G
    for k in range(1, K + 1):
        s = 1 << (K - k)
        ebk = (MULTS[2] if k == K else MULTS[1] if k == K - 1 else MULTS[0]) * eb
        fine = np.ascontiguousarray(field[::s, ::s, ::s])
        q, u, c, dec = po.level_encode(fine, coarse, ebk, RADIUS, use_ref=True)
        out[f"L{k}_codes"] = q.astype(np.uint16)
        out[f"L{k}_unpred"] = u
        out[f"L{k}_counts"] = c
        out[f"L{k}_eb"] = np.float64(ebk)
        if k < K:
            out[f"L{k}_encoder_grid"] = dec
        coarse = dec
    # reference decoder
    coarse = G
    for k in range(1, K + 1):
        q = out[f"L{k}_codes"].astype(np.int32).reshape(-1)
        dq = po.ref_dequantize(q, float(out[f"L{k}_eb"]), RADIUS, out[f"L{k}_unpred"], field.dtype)
        coarse = po.ref_level_decode(dq, coarse, 1 if k == K else 0)
        out[f"L{k}_decoded"] = coarse
    return out


def main():
    if not po.ref_available():
        po.build(ref=True)
    cases = {
        "grf32": (fields.grf((32, 32, 32), 11.0 / 3.0, 11, np.float32), 1e-3),
        "logn32": (fields.lognormal((32, 32, 32), 12, np.float32), 1e-4),
        "fronts64": (fields.fronts((16, 24, 32), 13, np.float64), 1e-6),
        "flat32": (np.full((16, 16, 16), 1e-3, dtype=np.float32), 1e-3),
    }
    arrays = {}
    for name, (f, rel) in cases.items():
        arrays[f"{name}_field"] = f
        arrays[f"{name}_rel"] = np.float64(rel)
        for k, v in hierarchy(f, rel).items():
            arrays[f"{name}_{k}"] = v
    # plain tricubic predictor of src/stz-rd.cpp (= src/float.cpp / double.cpp):
    # diff = sub - P for every block on a random reference grid with a flat half
    R = po.rd()
    rng = np.random.default_rng(8)
    for dt, suf in ((np.float32, "f32"), (np.float64, "f64")):
        dims = (9, 10, 12)
        ref = rng.standard_normal(dims).astype(dt)
        ref[:4] = 0.001
        sub = rng.standard_normal(dims).astype(dt)
        arrays[f"plain_{suf}_ref"] = ref
        arrays[f"plain_{suf}_sub"] = sub
        diffs = []
        for b in range(7):
            d = np.zeros(dims, dt)
            getattr(R, "rdref_preprocess_block_" + suf)(b, po._p(sub), po._p(ref), po._p(d), dims[2], dims[1], dims[0])
            diffs.append(d)
        arrays[f"plain_{suf}_diff"] = np.stack(diffs)

    # staged predictor of src/dependency.cpp (its stage functions, with FD5's
    # quantizer, split and merge, through the hierarchy; chunks 8 / 4, level
    # multipliers 1 / 2.5 / 6.25): each level's chunk-major codes per block
    # and the decoded field
    f = fields.grf((32, 32, 32), 3.0, 21, np.float32)
    eb = po.pointwise_eb(f, 1e-3, (1.0, 2.5, 6.25))
    st = po.ref_round_trip_staged(f, eb, (1.0, 2.5, 6.25), chunk_high=8, chunk_low=4)
    arrays["staged_field"] = f
    arrays["staged_eb"] = np.float64(eb)
    arrays["staged_K"] = np.int64(st["K"])
    for k in range(1, st["K"] + 1):
        arrays[f"staged_L{k}_codes"] = np.stack(st["codes"][k - 1])
    arrays["staged_decoded"] = st["grids"][st["K"]]
    # 12-point truncated bicubic of src/stz2.cpp, the same way
    tr = po.ref_round_trip_trunc(f, eb, (1.0, 2.5, 6.25), chunk_high=8, chunk_low=4)
    for k in range(1, tr["K"] + 1):
        arrays[f"trunc_L{k}_codes"] = np.stack(tr["codes"][k - 1])
    arrays["trunc_decoded"] = tr["grids"][tr["K"]]

    rng = np.random.default_rng(5)
    plans, offs, queries = [], [0], []
    for dims, ch, cl in [((256, 256, 256), 32, 16), ((384, 384, 256), 32, 16)]:
        for t in range(60):
            a = rng.integers(-8, np.array(dims) + 8)
            b = rng.integers(-8, np.array(dims) + 8)
            if t % 4 == 0:
                ax = rng.integers(0, 3)
                b[ax] = a[ax]
            p = po.plan(dims, ch, cl, a, b, use_ref=True)
            plans.append(p)
            offs.append(offs[-1] + p.size)
            queries.append([*dims, ch, cl, *a, *b])
    arrays["plan_queries"] = np.array(queries, dtype=np.int64)
    arrays["plan_offsets"] = np.array(offs, dtype=np.int64)
    arrays["plan_records"] = np.concatenate(plans)
    path = os.path.join(HERE, "fd5_golden.npz")
    np.savez_compressed(path, **arrays)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
