"""ctypes bindings of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Two libraries:
  * lib/libstz_oracle.so  the plain-C restatement (stz_oracle.c), built from
    committed sources by `make -C oracle oracle` (or __graft_entry__.build()).
  * _ref/libfd5ref.so     the reference's own FD5 translation unit compiled from
    its sources (`make -C oracle ref`, only where the reference is mounted;
    the built file travels with the repository snapshot).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "libstz_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libfd5ref.so")
# The reference's src/ directory, from the environment (no default: the
# reference sources exist only where the caller says they are).
REFERENCE_SRC = os.environ.get("STZ_REFERENCE_SRC", "")

vp, sz, dbl, ci = C.c_void_p, C.c_size_t, C.c_double, C.c_int


class Model(C.Structure):
    """stzo_model: int8 MLP 14 -> 32 -> 32 -> 7 of one level (the container's
    2112-byte layout)."""
    _fields_ = [("s_in", dbl), ("s_out", dbl), ("w1", (C.c_int8 * 16) * 32), ("b1", C.c_int32 * 32),
                ("m1", C.c_int32), ("sh1", C.c_int32), ("w2", (C.c_int8 * 32) * 32), ("b2", C.c_int32 * 32),
                ("m2", C.c_int32), ("sh2", C.c_int32), ("w3", (C.c_int8 * 32) * 8), ("b3", C.c_int32 * 8)]


class Params(C.Structure):
    _fields_ = [("dtype", ci), ("predictor", ci), ("radius", ci), ("chunk_high", ci), ("chunk_low", ci),
                ("zstd_level", ci), ("eb", dbl), ("mult_base", dbl), ("mult_low", dbl), ("mult_high", dbl),
                ("model", C.POINTER(Model) * 2), ("learned_flags", C.c_uint32 * 2)]


def model_record(m: Model) -> bytes:
    return C.string_at(C.addressof(m), C.sizeof(m))


def mlp_corr(m: Model, coarse: np.ndarray, x: int, y: int, z: int, eb: float) -> np.ndarray:
    """Corrections of the 7 blocks at interior coarse point (x, y, z)."""
    L = oracle()
    a = np.ascontiguousarray(coarse)
    dz, dy, dx = a.shape
    out = np.zeros(7, dtype=a.dtype)
    fn = L.stzo_mlp_corr_f64 if a.dtype == np.float64 else L.stzo_mlp_corr_f32
    fn(C.byref(m), _p(a), x, y, z, dx, dy, dz, C.c_double(eb), _p(out))
    return out


def build(ref: bool = True, reference_src: str | None = None) -> None:
    """Compile the oracle, and the reference shim when `reference_src` (default
    $STZ_REFERENCE_SRC) names a directory holding the reference's sources."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    src = reference_src if reference_src is not None else REFERENCE_SRC
    if ref and src and os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE_SRC={src}"], check=True)


_orc = None
_ref = None


def oracle() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        L.stzo_compress.restype = C.c_longlong
        L.stzo_compress.argtypes = [vp, ci, ci, ci, C.POINTER(Params), C.POINTER(C.POINTER(C.c_uint8))]
        L.stzo_decompress.argtypes = [vp, sz, ci, vp, C.POINTER(ci)]
        L.stzo_decompress_box.argtypes = [vp, sz, C.POINTER(ci), C.POINTER(ci), vp]
        L.stzo_stream_info.argtypes = [vp, sz, C.POINTER(ci), C.POINTER(ci), C.POINTER(ci)]
        L.stzo_debug_stream_codes.restype = C.c_longlong
        L.stzo_debug_stream_codes.argtypes = [vp, sz, ci, ci, vp, sz]
        L.stzo_free.argtypes = [vp]
        L.stzo_plan.restype = C.c_longlong
        L.stzo_plan.argtypes = [ci] * 11 + [vp, C.c_longlong]
        L.stzo_codebook.argtypes = [vp, ci, vp, vp]
        for suf in ("f32", "f64"):
            getattr(L, "stzo_level_encode_" + suf).argtypes = [vp, vp, ci, ci, ci, ci, dbl, ci, vp, vp, sz, vp, vp]
            getattr(L, "stzo_level_decode_" + suf).argtypes = [vp, vp, vp, vp, ci, ci, ci, ci, dbl, ci, vp]
            getattr(L, "stzo_quantize_" + suf).restype = C.c_longlong
            getattr(L, "stzo_quantize_" + suf).argtypes = [vp, sz, dbl, ci, vp, vp, sz]
            getattr(L, "stzo_predict_" + suf).argtypes = [ci, vp, ci, ci, ci, ci, ci, ci]
            getattr(L, "stzo_predict_plain_" + suf).argtypes = [ci, vp, ci, ci, ci, ci, ci, ci]
        L.stzo_predict_f32.restype = C.c_float
        L.stzo_predict_plain_f32.restype = C.c_float
        L.stzo_predict_f64.restype = C.c_double
        L.stzo_predict_plain_f64.restype = C.c_double
        L.stzo_num_levels.argtypes = [ci, ci, ci]
        L.stzo_level_chunk.argtypes = [ci] * 6
        _orc = L
    return _orc


RD_SO = os.path.join(HERE, "_ref", "libstzrd_ref.so")
_rd = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def rd_available() -> bool:
    return os.path.exists(RD_SO)


def rd() -> C.CDLL:
    """The reference's plain tricubic variant (src/stz-rd.cpp) compiled from source."""
    global _rd
    if _rd is None:
        L = C.CDLL(RD_SO)
        for suf in ("f32", "f64"):
            getattr(L, "rdref_preprocess_block_" + suf).argtypes = [ci, vp, vp, vp, ci, ci, ci]
            getattr(L, "rdref_depreprocess_block_" + suf).argtypes = [ci, vp, vp, vp] + [ci] * 9
        _rd = L
    return _rd


DEP_SO = os.path.join(HERE, "_ref", "libdep_ref.so")
_dep = None


def dep_available() -> bool:
    return os.path.exists(DEP_SO)


def dep() -> C.CDLL:
    """The reference's staged-predictor experiment (src/dependency.cpp, float
    only) compiled from source: its four stage functions."""
    global _dep
    if _dep is None:
        L = C.CDLL(DEP_SO)
        for f in ("depref_preprocess_block", "depref_depreprocess_block"):
            getattr(L, f).argtypes = [ci, vp, vp, vp, ci, ci, ci]
        for f in ("depref_preprocess_block_staged", "depref_depreprocess_block_staged"):
            getattr(L, f).argtypes = [ci, vp, vp, vp, ci, ci, ci]
        _dep = L
    return _dep


STZ2_SO = os.path.join(HERE, "_ref", "libstz2_ref.so")
_stz2 = None


def stz2_available() -> bool:
    return os.path.exists(STZ2_SO)


def stz2() -> C.CDLL:
    """The reference's 12-point truncated bicubic experiment (src/stz2.cpp,
    float only) compiled from source: preprocess_block / depreprocess_block."""
    global _stz2
    if _stz2 is None:
        L = C.CDLL(STZ2_SO)
        for f in ("stz2ref_preprocess_block", "stz2ref_depreprocess_block"):
            getattr(L, f).argtypes = [ci, vp, vp, vp, ci, ci, ci]
        _stz2 = L
    return _stz2


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        for suf in ("f32", "f64"):
            getattr(L, "fd5ref_level_encode_" + suf).argtypes = [vp, vp, ci, ci, ci, dbl, ci, vp, vp, sz, vp, vp]
            getattr(L, "fd5ref_level_decode_" + suf).argtypes = [vp, vp, ci, ci, ci, ci, vp]
            getattr(L, "fd5ref_dequantize_" + suf).argtypes = [vp, sz, dbl, ci, vp, vp]
            getattr(L, "fd5ref_quantize_range_nodec_" + suf).restype = C.c_longlong
            getattr(L, "fd5ref_quantize_range_nodec_" + suf).argtypes = [vp, sz, dbl, ci, vp, vp, sz]
            getattr(L, "fd5ref_preprocess_block_zslab_" + suf).argtypes = [ci, vp, vp, vp] + [ci] * 5
            getattr(L, "fd5ref_depreprocess_block_zslab_" + suf).argtypes = [ci, vp, vp, vp] + [ci] * 5
            getattr(L, "fd5ref_depreprocess_block_zslab_to_full_" + suf).argtypes = [ci, vp, vp, vp] + [ci] * 5
            getattr(L, "fd5ref_depreprocess_block_roi_" + suf).argtypes = [ci, vp, vp, vp] + [ci] * 9
            getattr(L, "fd5ref_slice_full_data_" + suf).argtypes = [vp, vp, ci, ci, ci]
            getattr(L, "fd5ref_merge_sub_blocks_to_full_" + suf).argtypes = [vp, vp, ci, ci, ci]
        L.fd5ref_plan.restype = C.c_longlong
        L.fd5ref_plan.argtypes = [ci] * 11 + [vp, C.c_longlong]
        _ref = L
    return _ref


def _p(a):
    return a.ctypes.data_as(vp)


def _suf(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


# ---- hierarchy shape -------------------------------------------------------
def num_levels(nx, ny, nz) -> int:
    return oracle().stzo_num_levels(nx, ny, nz)


def pointwise_eb(field: np.ndarray, rel: float, mults=(0.7, 2.7, 8.2)) -> float:
    """eb the library uses for a relative, pointwise bound (value range as
    computeRange, FD5:92-104)."""
    rng = float(field.max()) - float(field.min())
    E = rel * rng
    if not (E > 0):
        E = rel
    return E / max(mults)


# ---- whole-field codec -------------------------------------------------------
def compress(field: np.ndarray, eb: float, predictor=0, radius=32768, chunk_high=32, chunk_low=16, zstd_level=3,
             mults=(0.7, 2.7, 8.2), models=(None, None), flags=(0, 0)) -> bytes:
    """models / flags: learned correction of levels K-1 and K (Model or None,
    block bit masks)."""
    L = oracle()
    a = np.ascontiguousarray(field)
    nz, ny, nx = a.shape
    p = Params(1 if a.dtype == np.float64 else 0, predictor, radius, chunk_high, chunk_low, zstd_level, eb, *mults)
    for i in range(2):
        p.model[i] = C.pointer(models[i]) if models[i] is not None else C.POINTER(Model)()
        p.learned_flags[i] = int(flags[i]) if models[i] is not None else 0
    out = C.POINTER(C.c_uint8)()
    n = L.stzo_compress(_p(a), nx, ny, nz, C.byref(p), C.byref(out))
    if n < 0:
        raise ValueError(f"oracle compress failed ({n})")
    b = C.string_at(out, n)
    L.stzo_free(out)
    return b


def info(stream: bytes):
    L = oracle()
    dt, K = ci(), ci()
    dims = (ci * 3)()
    rc = L.stzo_stream_info(stream, len(stream), C.byref(dt), dims, C.byref(K))
    if rc:
        raise ValueError(f"bad stream ({rc})")
    return (np.float64 if dt.value else np.float32), (dims[2], dims[1], dims[0]), K.value


def decompress(stream: bytes, level: int = 0) -> np.ndarray:
    L = oracle()
    dt, (nz, ny, nx), K = info(stream)
    out = np.empty((nz >> level, ny >> level, nx >> level), dtype=dt)
    od = (ci * 3)()
    rc = L.stzo_decompress(stream, len(stream), level, _p(out), od)
    if rc:
        raise ValueError(f"oracle decompress failed ({rc})")
    return out


def decompress_box(stream: bytes, lo, hi) -> np.ndarray:
    L = oracle()
    dt, (nz, ny, nx), K = info(stream)
    dims = [nx, ny, nz]
    ext = []
    for ax in range(3):
        a, b = int(lo[ax]), int(hi[ax])
        if a == b:
            ext.append(1)
        else:
            l_ = max(0, min(a, b))
            h_ = min(dims[ax] - 1, max(a, b))
            ext.append(max(h_, l_) - l_ + 1)
    out = np.empty((ext[2], ext[1], ext[0]), dtype=dt)
    rc = L.stzo_decompress_box(stream, len(stream), (ci * 3)(*lo), (ci * 3)(*hi), _p(out))
    if rc:
        raise ValueError(f"oracle box decode failed ({rc})")
    return out


def stream_codes(stream: bytes, k: int, block: int) -> np.ndarray:
    L = oracle()
    _, (nz, ny, nx), _ = info(stream)
    buf = np.empty(nx * ny * nz, dtype=np.uint16)
    n = L.stzo_debug_stream_codes(stream, len(stream), k, block, _p(buf), buf.size)
    if n < 0:
        raise ValueError(f"oracle stream decode failed ({n})")
    return buf[:n].copy()


def codebook(hist: np.ndarray):
    L = oracle()
    h = np.ascontiguousarray(hist, dtype=np.uint32)
    sym = np.zeros(len(h), dtype=np.uint16)
    ln = np.zeros(len(h), dtype=np.uint8)
    n = L.stzo_codebook(_p(h), len(h), _p(sym), _p(ln))
    return sym[:n].copy(), ln[:n].copy()


def run_slots(hist: np.ndarray, plane: int):
    L = oracle()
    h = np.ascontiguousarray(hist, dtype=np.uint32)
    base = C.c_uint32()
    n = L.stzo_run_slots(_p(h), len(h), int(plane), C.byref(base))
    return base.value, n


# ---- level functions -----------------------------------------------------------
def level_encode(fine, coarse, eb, radius=32768, predictor=0, decoded=True, use_ref=False):
    """Codes (7, n) row-major per block, unpred values, counts, decoded fine grid."""
    dz, dy, dx = coarse.shape
    n = dx * dy * dz
    q = np.zeros(7 * n, dtype=np.int32)
    u = np.zeros(7 * n, dtype=coarse.dtype)
    c = np.zeros(7, dtype=np.uint64)
    d = np.zeros(fine.shape, dtype=coarse.dtype) if decoded else None
    fine = np.ascontiguousarray(fine)
    coarse = np.ascontiguousarray(coarse)
    suf = _suf(coarse.dtype)
    if use_ref:
        if predictor != 0:
            raise ValueError("the FD5 reference has only the dynamic predictor")
        rc = getattr(ref(), "fd5ref_level_encode_" + suf)(_p(fine), _p(coarse), dx, dy, dz, eb, radius, _p(q), _p(u),
                                                           u.size, _p(c), _p(d) if d is not None else None)
    else:
        rc = getattr(oracle(), "stzo_level_encode_" + suf)(_p(fine), _p(coarse), dx, dy, dz, predictor, eb, radius,
                                                            _p(q), _p(u), u.size, _p(c), _p(d) if d is not None else None)
    if rc:
        raise ValueError("level encode failed")
    return q.reshape(7, n), u[: int(c.sum())].copy(), c, d


def ref_level_decode(dq7: np.ndarray, coarse: np.ndarray, mode: int) -> np.ndarray:
    dz, dy, dx = coarse.shape
    out = np.zeros((2 * dz, 2 * dy, 2 * dx), dtype=coarse.dtype)
    getattr(ref(), "fd5ref_level_decode_" + _suf(coarse.dtype))(_p(np.ascontiguousarray(dq7)), _p(coarse), dx, dy, dz,
                                                                mode, _p(out))
    return out


def ref_dequantize(q: np.ndarray, eb: float, radius: int, unpred: np.ndarray, dtype) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.int32)
    out = np.zeros(q.size, dtype=dtype)
    un = np.ascontiguousarray(unpred, dtype=dtype)
    getattr(ref(), "fd5ref_dequantize_" + _suf(dtype))(_p(q), q.size, eb, radius, _p(un), _p(out))
    return out


def ref_round_trip(field: np.ndarray, eb: float, mults=(0.7, 2.7, 8.2), radius: int = 32768,
                   chunk_high: int = 32, chunk_low: int = 16) -> dict:
    """The reference's own FD5 level functions (oracle/_ref) driven through
    this project's hierarchy, for full-size parity checks.

    Encoder: per level k = 1..K the reference's predict + quantize of the 7
    odd-parity blocks against the encoder's decoded coarser grid, with the
    closed loop of FD5:2195-2230 (the decoded fine grid feeds level k + 1);
    level eb = multiplier x eb (base / low / high, FD5:2120-2129). Decoder:
    the reference's dequantize (recover LUT and row-major unpredictable
    values, FD5:1528-1562) and level decode (FD5:2369-2394 for the coarser
    levels, the fused to-full path FD5:2413-2451 for the finest).

    Returns codes[k-1] as the container's chunk-major uint16 symbols per block
    (7 arrays), unpred[k-1] counts per block, grids[j] = the decoder's grid
    after j levels (grids[0] the raw coarsest grid, grids[K] the field), and
    closed_loop_ok: every encoder-side decoded grid equals the decoder's."""
    a = np.ascontiguousarray(field)
    nz, ny, nx = a.shape
    K = num_levels(nx, ny, nz)
    S = 1 << K
    coarsest = np.ascontiguousarray(a[::S, ::S, ::S])
    enc_grid, dec_grid = coarsest, coarsest
    grids, codes, unpred = [coarsest], [], []
    closed_loop_ok = True
    for k in range(1, K + 1):
        s = 1 << (K - k)
        fine = a if s == 1 else np.ascontiguousarray(a[::s, ::s, ::s])
        ebk = (mults[2] if k == K else mults[1] if k == K - 1 else mults[0]) * eb
        q, u, c, d = level_encode(fine, enc_grid, ebk, radius, decoded=k < K, use_ref=True)
        dz, dy, dx = enc_grid.shape
        C_ = oracle().stzo_level_chunk(nx, ny, nz, k, chunk_high, chunk_low)
        codes.append([chunk_major(q[b], (dz, dy, dx), C_).astype(np.uint16) for b in range(7)])
        unpred.append([int(v) for v in c])
        dq = ref_dequantize(q.reshape(-1), ebk, radius, u, a.dtype)
        dec_grid = ref_level_decode(dq, dec_grid, 1 if k == K else 0)
        grids.append(dec_grid)
        if k < K:
            closed_loop_ok &= bool(np.array_equal(d.view(np.uint8), dec_grid.view(np.uint8)))
            enc_grid = d
    return {"K": K, "codes": codes, "unpred": unpred, "grids": grids, "closed_loop_ok": closed_loop_ok}


def ref_round_trip_plain(field: np.ndarray, eb: float, mults=(1.0, 2.5, 6.25), radius: int = 32768,
                         chunk_high: int = 32, chunk_low: int = 16) -> dict:
    """The plain tricubic pipeline of the reference's artifact programs
    (src/float.cpp / src/double.cpp main: preprocess_block on each level's
    7 odd-parity sub-blocks against the decoded coarser grid, the linear
    quantizer at multiplier x eb with multipliers 1 / 2.5 / 6.25 for base /
    low / high, float.cpp:598, 634, 706; decode by depreprocess_block and
    merge_sub_blocks_to_full), with the predictor from src/stz-rd.cpp and the
    quantizer, dequantizer and merge from FD5, all compiled from source
    (oracle/_ref), driven through this project's hierarchy. Returns the same
    record as ref_round_trip."""
    a = np.ascontiguousarray(field)
    nz, ny, nx = a.shape
    K = num_levels(nx, ny, nz)
    S = 1 << K
    suf = _suf(a.dtype)
    R, D = ref(), rd()
    grid = np.ascontiguousarray(a[::S, ::S, ::S])
    grids, codes, unpred = [grid], [], []
    for k in range(1, K + 1):
        s = 1 << (K - k)
        fine = a if s == 1 else np.ascontiguousarray(a[::s, ::s, ::s])
        ebk = (mults[2] if k == K else mults[1] if k == K - 1 else mults[0]) * eb
        dz, dy, dx = grid.shape
        n = dx * dy * dz
        C_ = oracle().stzo_level_chunk(nx, ny, nz, k, chunk_high, chunk_low)
        subs = np.empty((8, dz, dy, dx), a.dtype)
        getattr(R, "fd5ref_slice_full_data_" + suf)(_p(fine), _p(subs), 2 * dx, 2 * dy, 2 * dz)
        out = np.empty((8, dz, dy, dx), a.dtype)
        out[0] = grid
        lc, lu = [], []
        for b in range(7):
            diff = np.empty((dz, dy, dx), a.dtype)
            getattr(D, "rdref_preprocess_block_" + suf)(b, _p(subs[b + 1]), _p(grid), _p(diff), dx, dy, dz)
            q = np.empty(n, np.int32)
            u = np.empty(n, a.dtype)
            nu = getattr(R, "fd5ref_quantize_range_nodec_" + suf)(_p(diff), n, ebk, radius, _p(q), _p(u), n)
            lc.append(chunk_major(q, (dz, dy, dx), C_).astype(np.uint16))
            lu.append(int(nu))
            dq = ref_dequantize(q, ebk, radius, u[:nu], a.dtype).reshape(dz, dy, dx)
            getattr(D, "rdref_depreprocess_block_" + suf)(b, _p(dq), _p(grid), _p(out[b + 1]), dx, dy, dz, dx, dy,
                                                           dz, 0, 0, 0)
        nxt = np.empty((2 * dz, 2 * dy, 2 * dx), a.dtype)
        getattr(R, "fd5ref_merge_sub_blocks_to_full_" + suf)(_p(out), _p(nxt), dx, dy, dz)
        codes.append(lc)
        unpred.append(lu)
        grid = nxt
        grids.append(grid)
    return {"K": K, "codes": codes, "unpred": unpred, "grids": grids, "closed_loop_ok": True}


def ref_round_trip_staged(field: np.ndarray, eb: float, mults=(1.0, 2.5, 6.25), radius: int = 32768,
                          chunk_high: int = 32, chunk_low: int = 16) -> dict:
    """The staged pipeline of src/dependency.cpp (float only): per level,
    blocks 0, 1, 3 through preprocess_block against the decoded coarser grid,
    then 2, 4, 5 and last 6 through preprocess_block_staged against the
    decoded siblings, each block's residuals quantized (FD5's
    quantize_range_nodec at multiplier x eb, multipliers 1 / 2.5 / 6.25 as
    dependency.cpp:602, 674) and its decoded values rebuilt by the matching
    depreprocess function before the next stage reads them
    (dependency.cpp:591-634, 659-704); merge_sub_blocks_to_full builds the next
    level's grid. Stage functions from dependency.cpp, quantizer, dequantizer,
    split and merge from FD5, all compiled from source (oracle/_ref), driven
    through this project's hierarchy. Returns the same record as
    ref_round_trip."""
    a = np.ascontiguousarray(field)
    if a.dtype != np.float32:
        raise ValueError("src/dependency.cpp is float only")
    nz, ny, nx = a.shape
    K = num_levels(nx, ny, nz)
    S = 1 << K
    R, D = ref(), dep()
    grid = np.ascontiguousarray(a[::S, ::S, ::S])
    grids, codes, unpred = [grid], [], []
    for k in range(1, K + 1):
        s = 1 << (K - k)
        fine = a if s == 1 else np.ascontiguousarray(a[::s, ::s, ::s])
        ebk = (mults[2] if k == K else mults[1] if k == K - 1 else mults[0]) * eb
        dz, dy, dx = grid.shape
        n = dx * dy * dz
        C_ = oracle().stzo_level_chunk(nx, ny, nz, k, chunk_high, chunk_low)
        subs = np.empty((8, dz, dy, dx), a.dtype)
        R.fd5ref_slice_full_data_f32(_p(fine), _p(subs), 2 * dx, 2 * dy, 2 * dz)
        out = np.zeros((8, dz, dy, dx), a.dtype)
        out[0] = grid
        # ref_x, ref_y, ref_z, ref_xy, ref_xz, ref_yz: sub-blocks 1, 2, 4, 3, 5, 6
        refs = (C.c_void_p * 6)(*[out[i].ctypes.data for i in (1, 2, 4, 3, 5, 6)])
        lc, lu = [None] * 7, [0] * 7
        for b in (0, 1, 3, 2, 4, 5, 6):
            diff = np.empty((dz, dy, dx), a.dtype)
            if b in (0, 1, 3):
                D.depref_preprocess_block(b, _p(subs[b + 1]), _p(grid), _p(diff), dx, dy, dz)
            else:
                D.depref_preprocess_block_staged(b, _p(subs[b + 1]), refs, _p(diff), dx, dy, dz)
            q = np.empty(n, np.int32)
            u = np.empty(n, a.dtype)
            nu = R.fd5ref_quantize_range_nodec_f32(_p(diff), n, ebk, radius, _p(q), _p(u), n)
            lc[b] = chunk_major(q, (dz, dy, dx), C_).astype(np.uint16)
            lu[b] = int(nu)
            dq = ref_dequantize(q, ebk, radius, u[:nu], a.dtype).reshape(dz, dy, dx)
            if b in (0, 1, 3):
                D.depref_depreprocess_block(b, _p(dq), _p(grid), _p(out[b + 1]), dx, dy, dz)
            else:
                D.depref_depreprocess_block_staged(b, _p(dq), refs, _p(out[b + 1]), dx, dy, dz)
        nxt = np.empty((2 * dz, 2 * dy, 2 * dx), a.dtype)
        R.fd5ref_merge_sub_blocks_to_full_f32(_p(out), _p(nxt), dx, dy, dz)
        codes.append(lc)
        unpred.append(lu)
        grid = nxt
        grids.append(grid)
    return {"K": K, "codes": codes, "unpred": unpred, "grids": grids, "closed_loop_ok": True}


def ref_round_trip_trunc(field: np.ndarray, eb: float, mults=(1.0, 2.5, 6.25), radius: int = 32768,
                         chunk_high: int = 32, chunk_low: int = 16) -> dict:
    """The pipeline of src/stz2.cpp (float only): per level, its
    preprocess_block on the 7 odd-parity sub-blocks against the decoded
    coarser grid, FD5's quantize_range_nodec at multiplier x eb (multipliers
    1 / 2.5 / 6.25, stz2.cpp:694, 766), its depreprocess_block on the
    dequantized residuals, merge_sub_blocks_to_full; stz2.cpp's functions and
    FD5's quantizer, dequantizer, split and merge compiled from source
    (oracle/_ref), driven through this project's hierarchy. Returns the same
    record as ref_round_trip."""
    a = np.ascontiguousarray(field)
    if a.dtype != np.float32:
        raise ValueError("src/stz2.cpp is float only")
    nz, ny, nx = a.shape
    K = num_levels(nx, ny, nz)
    S = 1 << K
    R, D = ref(), stz2()
    grid = np.ascontiguousarray(a[::S, ::S, ::S])
    grids, codes, unpred = [grid], [], []
    for k in range(1, K + 1):
        s = 1 << (K - k)
        fine = a if s == 1 else np.ascontiguousarray(a[::s, ::s, ::s])
        ebk = (mults[2] if k == K else mults[1] if k == K - 1 else mults[0]) * eb
        dz, dy, dx = grid.shape
        n = dx * dy * dz
        C_ = oracle().stzo_level_chunk(nx, ny, nz, k, chunk_high, chunk_low)
        subs = np.empty((8, dz, dy, dx), a.dtype)
        R.fd5ref_slice_full_data_f32(_p(fine), _p(subs), 2 * dx, 2 * dy, 2 * dz)
        out = np.empty((8, dz, dy, dx), a.dtype)
        out[0] = grid
        lc, lu = [], []
        for b in range(7):
            diff = np.empty((dz, dy, dx), a.dtype)
            D.stz2ref_preprocess_block(b, _p(subs[b + 1]), _p(grid), _p(diff), dx, dy, dz)
            q = np.empty(n, np.int32)
            u = np.empty(n, a.dtype)
            nu = R.fd5ref_quantize_range_nodec_f32(_p(diff), n, ebk, radius, _p(q), _p(u), n)
            lc.append(chunk_major(q, (dz, dy, dx), C_).astype(np.uint16))
            lu.append(int(nu))
            dq = ref_dequantize(q, ebk, radius, u[:nu], a.dtype).reshape(dz, dy, dx)
            D.stz2ref_depreprocess_block(b, _p(dq), _p(grid), _p(out[b + 1]), dx, dy, dz)
        nxt = np.empty((2 * dz, 2 * dy, 2 * dx), a.dtype)
        R.fd5ref_merge_sub_blocks_to_full_f32(_p(out), _p(nxt), dx, dy, dz)
        codes.append(lc)
        unpred.append(lu)
        grid = nxt
        grids.append(grid)
    return {"K": K, "codes": codes, "unpred": unpred, "grids": grids, "closed_loop_ok": True}


def plan(dims_xyz, chunk_high, chunk_low, a, b, use_ref=False) -> np.ndarray:
    out = np.zeros(1 << 20, dtype=np.int64)
    fn = ref().fd5ref_plan if use_ref else oracle().stzo_plan
    n = fn(*[int(v) for v in dims_xyz], chunk_high, chunk_low, *[int(v) for v in a], *[int(v) for v in b], _p(out),
           out.size)
    if n < 0:
        raise ValueError("plan failed")
    return out[:n].copy()


def chunk_major(q_rm: np.ndarray, dims_zyx, C_: int) -> np.ndarray:
    """Row-major block codes -> the container's chunk-major symbol order."""
    dz, dy, dx = dims_zyx
    a = q_rm.reshape(dz // C_, C_, dy // C_, C_, dx // C_, C_)
    return a.transpose(0, 2, 4, 1, 3, 5).reshape(-1)
