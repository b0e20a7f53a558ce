"""Python binding of the B200-native STZ library (libstz_b200.so) via ctypes.

The library is the product; this module only marshals arguments. It loads
the in-tree build (sc25-stz2_b200/lib/libstz_b200.so) and raises if it is
missing: there is no CPU fallback.

    ctx = Context(0)
    s = ctx.compress(field, eb=1e-3, eb_mode="rel")        # numpy or torch (CPU/CUDA)
    full = ctx.decompress(s)                                  # numpy array
    half = ctx.decompress(s, level=1)
    box = ctx.decompress_box(s, (0, 0, 0), (63, 63, 63))
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libstz_b200.so")

STZ_F32, STZ_F64 = 0, 1
_STATUS = {
    0: "ok", 1: "invalid argument", 2: "unsupported dimensions", 3: "CUDA error", 4: "out of memory",
    5: "invalid stream", 6: "zstd error", 7: "out of range", 8: "unsupported",
}


class StzError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class Opts(C.Structure):
    _fields_ = [
        ("eb", C.c_double), ("eb_mode", C.c_int), ("bound_mode", C.c_int),
        ("mult_base", C.c_double), ("mult_low", C.c_double), ("mult_high", C.c_double),
        ("radius", C.c_int), ("chunk_high", C.c_int), ("chunk_low", C.c_int),
        ("zstd_level", C.c_int), ("predictor", C.c_int), ("threads", C.c_int),
        ("model", C.c_void_p), ("learned_flags", C.c_int),
    ]


class Info(C.Structure):
    _fields_ = [
        ("dtype", C.c_int), ("predictor", C.c_int), ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
        ("n_levels", C.c_int), ("radius", C.c_int), ("chunk_high", C.c_int), ("chunk_low", C.c_int),
        ("eb", C.c_double), ("mult_base", C.c_double), ("mult_low", C.c_double), ("mult_high", C.c_double),
        ("max_error", C.c_double), ("stream_bytes", C.c_size_t), ("raw_payload_bytes", C.c_size_t),
        ("learned_flags", C.c_int),
    ]


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libstz_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libstz_b200.so not built: {path} is missing (run sc25-stz2_b200/build.py)")
    lib = C.CDLL(path)
    vp, sz, i64p = C.c_void_p, C.c_size_t, C.POINTER(C.c_int64)
    lib.stz_last_error.restype = C.c_char_p
    lib.stz_status_string.restype = C.c_char_p
    lib.stz_default_opts.argtypes = [C.POINTER(Opts)]
    lib.stz_context_create.argtypes = [C.c_int, C.POINTER(vp)]
    lib.stz_context_destroy.argtypes = [vp]
    lib.stz_context_sync.argtypes = [vp]
    for f in (lib.stz_compress, lib.stz_compress_dev):
        f.argtypes = [vp, vp, C.c_int, sz, sz, sz, C.POINTER(Opts), C.POINTER(vp)]
    for f in (lib.stz_decompress_full, lib.stz_decompress_full_dev):
        f.argtypes = [vp, vp, vp]
    for f in (lib.stz_decompress_level, lib.stz_decompress_level_dev):
        f.argtypes = [vp, vp, C.c_int, vp, C.POINTER(sz)]
    for f in (lib.stz_decompress_box, lib.stz_decompress_box_dev):
        f.argtypes = [vp, vp, i64p, i64p, vp, C.POINTER(sz)]
    lib.stz_stream_bytes.argtypes = [vp, C.POINTER(vp), C.POINTER(sz)]
    lib.stz_stream_parse.argtypes = [vp, vp, sz, C.POINTER(vp)]
    lib.stz_stream_info.argtypes = [vp, C.POINTER(Info)]
    lib.stz_stream_upload.argtypes = [vp, vp]
    lib.stz_stream_free.argtypes = [vp]
    lib.stz_stream_free.restype = None
    lib.stz_split_dev.argtypes = [vp, C.c_int, vp, sz, sz, sz, vp]
    lib.stz_merge_dev.argtypes = [vp, C.c_int, vp, sz, sz, sz, vp]
    for f in (lib.stz_preprocess_block_dev, lib.stz_depreprocess_block_dev, lib.stz_depreprocess_block_to_full_dev):
        f.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp] + [C.c_int] * 5
    lib.stz_depreprocess_block_roi_dev.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp] + [C.c_int] * 9
    for f in ("stz_preprocess_block_staged_dev", "stz_depreprocess_block_staged_dev"):
        getattr(lib, f).argtypes = [vp, C.c_int, C.c_int, vp, C.POINTER(vp), vp, C.c_size_t, C.c_size_t, C.c_size_t]
    lib.stz_quantize_dev.argtypes = [vp, C.c_int, vp, sz, C.c_double, C.c_int, vp, vp, C.POINTER(sz)]
    lib.stz_dequantize_dev.argtypes = [vp, C.c_int, vp, sz, C.c_double, C.c_int, vp, vp]
    lib.stz_plan_box.argtypes = [sz, sz, sz, C.c_int, C.c_int, i64p, i64p, i64p, sz, C.POINTER(sz)]
    lib.stz_debug_stream_codes.argtypes = [vp, vp, C.c_int, C.c_int, vp, sz, C.POINTER(sz)]
    lib.stz_debug_codebook.argtypes = [vp, C.c_int, vp, vp, C.POINTER(C.c_int)]
    lib.stz_debug_quant_table.argtypes = [C.c_double, C.c_int, vp, C.POINTER(C.c_float), C.POINTER(C.c_int)]
    lib.stz_debug_run_slots.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    lib.stz_quantize_noalloc_dev.argtypes = [C.c_int, vp, sz, C.c_double, C.c_int, vp, vp, C.POINTER(sz), vp]
    lib.stz_context_stream.argtypes = [vp, C.POINTER(vp)]
    lib.stz_profile_enable.argtypes = [vp, C.c_int]
    lib.stz_profile_reset.argtypes = [vp]
    lib.stz_profile_count.argtypes = [vp, C.POINTER(C.c_int)]
    lib.stz_profile_entry.argtypes = [vp, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                      C.POINTER(C.c_uint64)]
    lib.stz_server_default_opts.argtypes = [C.POINTER(ServerOpts)]
    lib.stz_server_default_opts.restype = None
    lib.stz_server_create.argtypes = [C.c_int, C.POINTER(ServerOpts), C.POINTER(vp)]
    lib.stz_server_destroy.argtypes = [vp]
    lib.stz_server_destroy.restype = None
    lib.stz_server_add_stream.argtypes = [vp, vp, sz, C.POINTER(C.c_int)]
    lib.stz_server_submit.argtypes = [vp, C.POINTER(Request), C.POINTER(C.c_uint64)]
    lib.stz_server_wait.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(Result)]
    lib.stz_server_copy_out.argtypes = [vp, C.c_uint64, vp]
    lib.stz_server_release.argtypes = [vp, C.c_uint64]
    lib.stz_server_stats_get.argtypes = [vp, C.POINTER(ServerStats)]
    lib.stz_server_batch_log.argtypes = [vp, C.POINTER(BatchRecord), sz, C.POINTER(sz)]
    lib.stz_default_train_opts.argtypes = [C.POINTER(TrainOpts)]
    lib.stz_default_train_opts.restype = None
    lib.stz_trainer_create.argtypes = [vp, C.POINTER(Opts), C.POINTER(TrainOpts), C.POINTER(vp)]
    lib.stz_trainer_add_field_dev.argtypes = [vp, vp, C.c_int, sz, sz, sz]
    lib.stz_trainer_fit.argtypes = [vp, C.POINTER(vp)]
    lib.stz_trainer_stats.argtypes = [vp, C.POINTER(TrainStats)]
    lib.stz_trainer_free.argtypes = [vp]
    lib.stz_trainer_free.restype = None
    lib.stz_debug_mlp_grad.argtypes = [vp, vp, vp, vp, sz, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.POINTER(C.c_double), vp, C.POINTER(C.c_double)]
    lib.stz_debug_learned_infer.argtypes = [vp, vp, sz, vp, C.c_int, vp]
    lib.stz_model_parse.argtypes = [vp, sz, C.POINTER(vp)]
    lib.stz_model_bytes.argtypes = [vp, C.POINTER(vp), C.POINTER(sz)]
    lib.stz_model_free.argtypes = [vp]
    lib.stz_model_free.restype = None
    _lib = lib
    return lib


class TrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int), ("qat_epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_double),
                ("huber_delta", C.c_double), ("sample_step", C.c_int), ("max_pairs", C.c_size_t),
                ("seed", C.c_uint64)]


class TrainStats(C.Structure):
    _fields_ = [("pairs", C.c_size_t * 2), ("loss_zero", C.c_double * 2), ("loss_float", C.c_double * 2),
                ("loss_qat", C.c_double * 2), ("loss_int8", C.c_double * 2), ("s_in", C.c_double * 2),
                ("s_t", C.c_double * 2), ("train_ms", C.c_double)]


class BatchRecord(C.Structure):
    _fields_ = [("batch", C.c_uint64), ("n_requests", C.c_int), ("lane", C.c_int), ("slot", C.c_int),
                ("t_start_ms", C.c_double),
                ("t_planned_ms", C.c_double), ("t_launched_ms", C.c_double), ("t_done_ms", C.c_double),
                ("device_ms", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("arena_bytes", C.c_size_t), ("max_batch", C.c_int), ("slots", C.c_int), ("autotune", C.c_int),
                ("threads", C.c_int), ("fast_reserve", C.c_size_t)]


class Request(C.Structure):
    _fields_ = [("stream_id", C.c_int), ("kind", C.c_int), ("lo", C.c_int64 * 3), ("hi", C.c_int64 * 3),
                ("level", C.c_int)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("out_dev", C.c_void_p), ("dims", C.c_size_t * 3), ("bytes", C.c_size_t),
                ("queue_ms", C.c_double), ("latency_ms", C.c_double), ("batch", C.c_uint64),
                ("batch_size", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("decode_grid", C.c_int), ("roi_block", C.c_int), ("roi_grid", C.c_int),
                ("arena_bytes", C.c_size_t), ("arena_in_use", C.c_size_t)]


def _check(status: int) -> None:
    if status != 0:
        raise StzError(status, _lib.stz_last_error().decode(errors="replace"))


def default_opts(**kw) -> Opts:
    lib = load_library()
    o = Opts()
    lib.stz_default_opts(C.byref(o))
    modes = {"abs": 0, "rel": 1}
    bounds = {"pointwise": 0, "reference": 1}
    preds = {"dynamic": 0, "cubic": 1, "staged": 2, "truncated": 3}
    for k, v in kw.items():
        if k == "eb_mode" and isinstance(v, str):
            v = modes[v]
        elif k == "bound_mode" and isinstance(v, str):
            v = bounds[v]
        elif k == "predictor" and isinstance(v, str):
            v = preds[v]
        elif k == "model":
            o._model_ref = v  # the model must outlive the options that point at it
            v = None if v is None else (v.handle.value if isinstance(v, Model) else v)
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def _dtype_code(dt) -> int:
    dt = np.dtype(dt)
    if dt == np.float32:
        return STZ_F32
    if dt == np.float64:
        return STZ_F64
    raise TypeError(f"unsupported dtype {dt}")


def _np_dtype(code: int):
    return np.float64 if code == STZ_F64 else np.float32


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _torch_sync(*ts) -> None:
    """The library works on its own CUDA stream: finish the work torch has
    queued on these tensors' devices before the library reads or writes them."""
    done = set()
    for t in ts:
        if t is not None and _is_torch(t) and t.is_cuda and t.device not in done:
            import torch

            torch.cuda.current_stream(t.device).synchronize()
            done.add(t.device)


@dataclass
class StreamInfo:
    dtype: type
    predictor: int
    shape: tuple  # (nz, ny, nx)
    n_levels: int
    radius: int
    chunk_high: int
    chunk_low: int
    eb: float
    mults: tuple
    max_error: float
    stream_bytes: int
    raw_payload_bytes: int
    learned_flags: int = 0  # bits 0-6: second-finest level's blocks, 8-14: finest level's


class Model:
    """Learned-correction models of the second-finest and finest levels
    (library-owned; the "STZLMDL1" file format of stz_model_parse)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_bytes(cls, data: bytes) -> "Model":
        lib = load_library()
        h = C.c_void_p()
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(lib.stz_model_parse(buf, len(data), C.byref(h)))
        return cls(h.value)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.stz_model_free(self._h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    def to_bytes(self) -> bytes:
        p, n = C.c_void_p(), C.c_size_t()
        _check(_lib.stz_model_bytes(self._h, C.byref(p), C.byref(n)))
        return C.string_at(p, n.value)


class Stream:
    """A compressed field (library-owned)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.stz_stream_free(self._h)
            self._h = C.c_void_p()

    @property
    def handle(self):
        return self._h

    def to_bytes(self) -> bytes:
        p, n = C.c_void_p(), C.c_size_t()
        _check(_lib.stz_stream_bytes(self._h, C.byref(p), C.byref(n)))
        return C.string_at(p, n.value)

    def __len__(self) -> int:
        p, n = C.c_void_p(), C.c_size_t()
        _check(_lib.stz_stream_bytes(self._h, C.byref(p), C.byref(n)))
        return n.value

    def info(self) -> StreamInfo:
        i = Info()
        _check(_lib.stz_stream_info(self._h, C.byref(i)))
        return StreamInfo(_np_dtype(i.dtype), i.predictor, (i.nz, i.ny, i.nx), i.n_levels, i.radius, i.chunk_high,
                          i.chunk_low, i.eb, (i.mult_base, i.mult_low, i.mult_high), i.max_error, i.stream_bytes,
                          i.raw_payload_bytes, i.learned_flags)


class Context:
    """One CUDA device + stream of the library."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self._c = C.c_void_p()
        _check(self.lib.stz_context_create(int(device), C.byref(self._c)))
        self.device = device

    def close(self):
        if self._c.value:
            self.lib.stz_context_destroy(self._c)
            self._c = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sync(self):
        _check(self.lib.stz_context_sync(self._c))

    def cuda_stream(self) -> int:
        """cudaStream_t of the context (as an integer handle)."""
        p = C.c_void_p()
        _check(self.lib.stz_context_stream(self._c, C.byref(p)))
        return p.value or 0

    def profile(self, on: bool = True) -> None:
        _check(self.lib.stz_profile_enable(self._c, 1 if on else 0))

    def profile_reset(self) -> None:
        _check(self.lib.stz_profile_reset(self._c))

    def profile_read(self) -> dict:
        """{kernel name: (total ms, launches)} since the last reset."""
        n = C.c_int()
        _check(self.lib.stz_profile_count(self._c, C.byref(n)))
        out = {}
        for i in range(n.value):
            name, ms, k = C.c_char_p(), C.c_double(), C.c_uint64()
            _check(self.lib.stz_profile_entry(self._c, i, C.byref(name), C.byref(ms), C.byref(k)))
            out[name.value.decode()] = (ms.value, k.value)
        return out

    # ---- codec -------------------------------------------------------------
    def compress(self, field, opts: Opts | None = None, **kw) -> Stream:
        """Compress a 3-D array (z, y, x) — numpy, or torch on CPU or CUDA."""
        o = opts if opts is not None else default_opts(**kw)
        h = C.c_void_p()
        if _is_torch(field):
            import torch

            if field.dim() != 3 or not field.is_contiguous():
                raise ValueError("field must be a contiguous 3-D tensor (z, y, x)")
            code = {torch.float32: STZ_F32, torch.float64: STZ_F64}[field.dtype]
            nz, ny, nx = field.shape
            _torch_sync(field)
            fn = self.lib.stz_compress_dev if field.is_cuda else self.lib.stz_compress
            _check(fn(self._c, C.c_void_p(field.data_ptr()), code, nx, ny, nz, C.byref(o), C.byref(h)))
        else:
            a = np.ascontiguousarray(field)
            if a.ndim != 3:
                raise ValueError("field must be 3-D (z, y, x)")
            nz, ny, nx = a.shape
            _check(self.lib.stz_compress(self._c, a.ctypes.data_as(C.c_void_p), _dtype_code(a.dtype), nx, ny, nz,
                                         C.byref(o), C.byref(h)))
        return Stream(h.value)

    def parse(self, data: bytes) -> Stream:
        h = C.c_void_p()
        buf = C.create_string_buffer(data, len(data))
        _check(self.lib.stz_stream_parse(self._c, buf, len(data), C.byref(h)))
        return Stream(h.value)

    def upload(self, s: Stream) -> None:
        _check(self.lib.stz_stream_upload(self._c, s.handle))

    def decompress(self, s: Stream, level: int = 0, out=None):
        """Full (level 0) or progressive decode. out: torch CUDA tensor for the
        device path, else a numpy array is returned."""
        inf = s.info()
        nz, ny, nx = inf.shape
        shape = (nz >> level, ny >> level, nx >> level)
        dims = (C.c_size_t * 3)()
        if out is not None and _is_torch(out) and out.is_cuda:
            if tuple(out.shape) != shape:
                raise ValueError(f"out must have shape {shape}")
            _torch_sync(out)
            _check(self.lib.stz_decompress_level_dev(self._c, s.handle, level, C.c_void_p(out.data_ptr()), dims))
            return out
        res = np.empty(shape, dtype=inf.dtype) if out is None else out
        _check(self.lib.stz_decompress_level(self._c, s.handle, level, res.ctypes.data_as(C.c_void_p), dims))
        return res

    def decompress_box(self, s: Stream, lo, hi, out=None):
        """Box / slice decode; lo, hi are inclusive (x, y, z) corners."""
        inf = s.info()
        a = (C.c_int64 * 3)(*[int(v) for v in lo])
        b = (C.c_int64 * 3)(*[int(v) for v in hi])
        nz, ny, nx = inf.shape
        dims = [nx, ny, nz]
        ext = []
        for ax in range(3):
            if a[ax] == b[ax]:
                ext.append(1)
            else:
                lo_ = max(0, min(a[ax], b[ax]))
                hi_ = min(dims[ax] - 1, max(a[ax], b[ax]))
                ext.append(max(hi_, lo_) - lo_ + 1)
        shape = (ext[2], ext[1], ext[0])
        od = (C.c_size_t * 3)()
        if out is not None and _is_torch(out) and out.is_cuda:
            _torch_sync(out)
            _check(self.lib.stz_decompress_box_dev(self._c, s.handle, a, b, C.c_void_p(out.data_ptr()), od))
            return out
        res = np.empty(shape, dtype=inf.dtype)
        _check(self.lib.stz_decompress_box(self._c, s.handle, a, b, res.ctypes.data_as(C.c_void_p), od))
        return res

    def stream_codes(self, s: Stream, level_from_coarse: int, block: int) -> np.ndarray:
        inf = s.info()
        n = C.c_size_t()
        cap = int(np.prod(inf.shape))
        buf = np.empty(cap, dtype=np.uint16)
        _check(self.lib.stz_debug_stream_codes(self._c, s.handle, level_from_coarse, block,
                                               buf.ctypes.data_as(C.c_void_p), cap, C.byref(n)))
        return buf[: n.value].copy()

    # ---- reference function boundary (torch CUDA tensors) ------------------
    # These entry points are asynchronous on the context's stream: inputs are
    # made ready first (_p), and outputs are ready after ctx.sync().
    def _p(self, t):
        _torch_sync(t)
        return C.c_void_p(t.data_ptr())

    def split(self, full, subs):
        nz, ny, nx = full.shape
        _check(self.lib.stz_split_dev(self._c, _tcode(full), self._p(full), nx, ny, nz, self._p(subs)))

    def merge(self, subs, full):
        _, hz, hy, hx = subs.shape
        _check(self.lib.stz_merge_dev(self._c, _tcode(full), self._p(subs), hx, hy, hz, self._p(full)))

    def preprocess_block(self, block, sub, ref, diff, z0=0, z1=None, predictor=0):
        dz, dy, dx = ref.shape
        _check(self.lib.stz_preprocess_block_dev(self._c, _tcode(ref), predictor, block, self._p(sub), self._p(ref),
                                                 self._p(diff), dx, dy, dz, z0, dz if z1 is None else z1))

    def depreprocess_block(self, block, de, ref, out, z0=0, z1=None, predictor=0):
        dz, dy, dx = ref.shape
        _check(self.lib.stz_depreprocess_block_dev(self._c, _tcode(ref), predictor, block, self._p(de), self._p(ref),
                                                   self._p(out), dx, dy, dz, z0, dz if z1 is None else z1))

    def depreprocess_block_to_full(self, block, de, ref, full, z0=0, z1=None, predictor=0):
        dz, dy, dx = ref.shape
        _check(self.lib.stz_depreprocess_block_to_full_dev(self._c, _tcode(ref), predictor, block, self._p(de),
                                                           self._p(ref), self._p(full), dx, dy, dz, z0,
                                                           dz if z1 is None else z1))

    def depreprocess_block_roi(self, block, de, ref, out, end, start, predictor=0):
        dz, dy, dx = ref.shape
        _check(self.lib.stz_depreprocess_block_roi_dev(self._c, _tcode(ref), predictor, block, self._p(de),
                                                       self._p(ref), self._p(out), dx, dy, dz, *end, *start))

    def _refs6(self, refs):
        return (C.c_void_p * 6)(*[None if r is None else self._p(r).value for r in (list(refs) + [None] * 6)[:6]])

    def preprocess_block_staged(self, block, sub, refs, diff):
        """dependency.cpp's stage functions: blocks 0, 1, 3 take refs = [coarse
        sub-block 0]; blocks 2, 4, 5, 6 take [ref_x, ref_y, ref_z, ref_xy,
        ref_xz, ref_yz] (None where the block does not read one)."""
        dz, dy, dx = sub.shape
        _check(self.lib.stz_preprocess_block_staged_dev(self._c, _tcode(sub), block, self._p(sub), self._refs6(refs),
                                                        self._p(diff), dx, dy, dz))

    def depreprocess_block_staged(self, block, de, refs, out):
        dz, dy, dx = de.shape
        _check(self.lib.stz_depreprocess_block_staged_dev(self._c, _tcode(de), block, self._p(de), self._refs6(refs),
                                                          self._p(out), dx, dy, dz))

    def quantize(self, data, eb, radius, q, unpred) -> int:
        n = C.c_size_t()
        _check(self.lib.stz_quantize_dev(self._c, _tcode(data), self._p(data), data.numel(), eb, radius, self._p(q),
                                         self._p(unpred), C.byref(n)))
        return n.value

    def dequantize(self, q, eb, radius, unpred, out):
        _check(self.lib.stz_dequantize_dev(self._c, _tcode(out), self._p(q), q.numel(), eb, radius, self._p(unpred),
                                           self._p(out)))


def quantize_noalloc(data, eb: float, radius: int, q, unpred, stream: int = 0) -> int:
    """Quantize CUDA tensors without any device allocation (no context needed):
    same results as Context.quantize, on the caller's stream, at most
    STZ_NOALLOC_MAX_VALUES values per call. Returns the unpredictable count."""
    lib = load_library()
    n = C.c_size_t()
    _check(lib.stz_quantize_noalloc_dev(_tcode(data), C.c_void_p(data.data_ptr()), data.numel(), eb, radius,
                                        C.c_void_p(q.data_ptr()), C.c_void_p(unpred.data_ptr()), C.byref(n),
                                        C.c_void_p(stream)))
    return n.value


NOALLOC_MAX_VALUES = 65536 * 1024

REQ_BOX, REQ_LEVEL = 0, 1


@dataclass
class ServedResult:
    ticket: int
    status: int
    out_dev: int  # device address (valid until release)
    shape: tuple  # (nz, ny, nx)
    nbytes: int
    queue_ms: float
    latency_ms: float
    batch: int
    batch_size: int


class Server:
    """Request server over streams resident on one GPU (stz_server_*):
    box / slice / progressive-level requests, continuously batched."""

    def __init__(self, device: int = 0, arena_bytes: int = 0, max_batch: int = 0, slots: int = 0,
                 autotune: bool = True, threads: int = 0, fast_reserve: int | None = None):
        self.lib = load_library()
        o = ServerOpts()
        self.lib.stz_server_default_opts(C.byref(o))
        if arena_bytes:
            o.arena_bytes = arena_bytes
        if max_batch:
            o.max_batch = max_batch
        if slots:
            o.slots = slots
        o.autotune = 1 if autotune else 0
        o.threads = threads
        if fast_reserve is not None:
            o.fast_reserve = fast_reserve
        self._s = C.c_void_p()
        _check(self.lib.stz_server_create(int(device), C.byref(o), C.byref(self._s)))

    def close(self):
        if self._s.value:
            self.lib.stz_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_stream(self, data) -> int:
        b = data.to_bytes() if isinstance(data, Stream) else bytes(data)
        sid = C.c_int()
        _check(self.lib.stz_server_add_stream(self._s, b, len(b), C.byref(sid)))
        return sid.value

    def _submit(self, r: Request) -> int:
        t = C.c_uint64()
        _check(self.lib.stz_server_submit(self._s, C.byref(r), C.byref(t)))
        return t.value

    def submit_box(self, stream_id: int, lo, hi) -> int:
        """lo/hi: inclusive (x, y, z) corners; lo == hi on one axis makes a slice."""
        r = Request()
        r.stream_id, r.kind = stream_id, REQ_BOX
        for a in range(3):
            r.lo[a], r.hi[a] = int(lo[a]), int(hi[a])
        return self._submit(r)

    def submit_level(self, stream_id: int, level: int) -> int:
        r = Request()
        r.stream_id, r.kind, r.level = stream_id, REQ_LEVEL, int(level)
        return self._submit(r)

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> ServedResult:
        r = Result()
        _check(self.lib.stz_server_wait(self._s, ticket, timeout_ms, C.byref(r)))
        return ServedResult(ticket, r.status, r.out_dev or 0, (r.dims[2], r.dims[1], r.dims[0]), r.bytes, r.queue_ms,
                            r.latency_ms, r.batch, r.batch_size)

    def copy_out(self, res: ServedResult, dtype=np.float32) -> np.ndarray:
        out = np.empty(res.shape, dtype=dtype)
        assert out.nbytes == res.nbytes, "dtype does not match the stream"
        _check(self.lib.stz_server_copy_out(self._s, res.ticket, out.ctypes.data_as(C.c_void_p)))
        return out

    def release(self, ticket: int) -> None:
        _check(self.lib.stz_server_release(self._s, ticket))

    def stats(self) -> dict:
        s = ServerStats()
        _check(self.lib.stz_server_stats_get(self._s, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def batch_log(self, cap: int = 4096) -> np.ndarray:
        """Recent batches, oldest first: columns batch, n_requests, lane, slot,
        t_start, t_planned, t_launched, t_done (ms since creation), device_ms."""
        recs = (BatchRecord * cap)()
        n = C.c_size_t()
        _check(self.lib.stz_server_batch_log(self._s, recs, cap, C.byref(n)))
        return np.array([[getattr(recs[i], f) for f, _ in BatchRecord._fields_] for i in range(n.value)],
                        dtype=np.float64).reshape(-1, len(BatchRecord._fields_))


def _tcode(t) -> int:
    import torch

    return {torch.float32: STZ_F32, torch.float64: STZ_F64}[t.dtype]


def plan_box(dims_xyz, chunk_high, chunk_low, a, b) -> np.ndarray:
    """ROI planner record (host-only, no GPU needed)."""
    lib = load_library()
    cap = 1 << 20
    out = np.zeros(cap, dtype=np.int64)
    n = C.c_size_t()
    aa = (C.c_int64 * 3)(*[int(v) for v in a])
    bb = (C.c_int64 * 3)(*[int(v) for v in b])
    _check(lib.stz_plan_box(*[int(d) for d in dims_xyz], chunk_high, chunk_low, aa, bb,
                            out.ctypes.data_as(C.POINTER(C.c_int64)), cap, C.byref(n)))
    return out[: n.value].copy()


def quant_table(eb: float, radius: int = 32768):
    """The f32 quantizer table of the plain level encoders (host only):
    (entries (64, 4) float32 {S_h, S_h+1, lo_h, hi_h}, r2, on)."""
    lib = load_library()
    e = np.zeros((64, 4), dtype=np.float32)
    r2, on = C.c_float(), C.c_int()
    _check(lib.stz_debug_quant_table(eb, radius, e.ctypes.data_as(C.c_void_p), C.byref(r2), C.byref(on)))
    return e, np.float32(r2.value), bool(on.value)


def codebook(hist: np.ndarray):
    """Canonical codebook of the container format (host-only)."""
    lib = load_library()
    h = np.ascontiguousarray(hist, dtype=np.uint32)
    sym = np.zeros(len(h), dtype=np.uint16)
    ln = np.zeros(len(h), dtype=np.uint8)
    n = C.c_int()
    _check(lib.stz_debug_codebook(h.ctypes.data_as(C.c_void_p), len(h), sym.ctypes.data_as(C.c_void_p),
                                  ln.ctypes.data_as(C.c_void_p), C.byref(n)))
    return sym[: n.value].copy(), ln[: n.value].copy()


def run_slots(hist: np.ndarray, plane: int):
    """(run_base, run_n) of the container's run symbols for a code histogram."""
    lib = load_library()
    h = np.ascontiguousarray(hist, dtype=np.uint32)
    base, n = C.c_uint32(), C.c_uint32()
    _check(lib.stz_debug_run_slots(h.ctypes.data_as(C.c_void_p), len(h), int(plane), C.byref(base), C.byref(n)))
    return base.value, n.value


class Trainer:
    """GPU training of the learned correction on pairs the compressor makes
    from the given fields (stz_trainer_*)."""

    def __init__(self, ctx: "Context", opts: Opts | None = None, train: TrainOpts | None = None, **kw):
        self.lib = load_library()
        self.ctx = ctx
        self.opts = opts if opts is not None else default_opts(**kw)
        self.train = train if train is not None else default_train_opts()
        self._h = C.c_void_p()
        _check(self.lib.stz_trainer_create(ctx._c, C.byref(self.opts), C.byref(self.train), C.byref(self._h)))

    def add_field(self, field) -> None:
        """field: a contiguous 3-D CUDA tensor (z, y, x), float32 or float64."""
        import torch

        if not (_is_torch(field) and field.is_cuda and field.dim() == 3 and field.is_contiguous()):
            raise ValueError("field must be a contiguous 3-D CUDA tensor (z, y, x)")
        code = {torch.float32: STZ_F32, torch.float64: STZ_F64}[field.dtype]
        nz, ny, nx = field.shape
        _torch_sync(field)
        _check(self.lib.stz_trainer_add_field_dev(self._h, C.c_void_p(field.data_ptr()), code, nx, ny, nz))

    def fit(self) -> Model:
        h = C.c_void_p()
        _check(self.lib.stz_trainer_fit(self._h, C.byref(h)))
        return Model(h.value)

    def stats(self) -> dict:
        st = TrainStats()
        _check(self.lib.stz_trainer_stats(self._h, C.byref(st)))
        out = {}
        for f, _ in TrainStats._fields_:
            v = getattr(st, f)
            out[f] = list(v) if hasattr(v, "__len__") else v
        return out

    def close(self) -> None:
        if self._h and self._h.value:
            self.lib.stz_trainer_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.stz_trainer_free(self._h)
            self._h = C.c_void_p()


def default_train_opts(**kw) -> TrainOpts:
    lib = load_library()
    t = TrainOpts()
    lib.stz_default_train_opts(C.byref(t))
    for k, v in kw.items():
        if not hasattr(t, k):
            raise TypeError(f"unknown training option {k}")
        setattr(t, k, v)
    return t


def mlp_grad(ctx: "Context", params, x, t, s_in: float, s_t: float, huber_delta: float = 2.0, qat: bool = False,
             sa=(1.0, 1.0)):
    """One forward + backward of the training kernels (stz_debug_mlp_grad):
    returns (mean loss, 1864 gradients)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    tt = np.ascontiguousarray(t, dtype=np.float32)
    n = xx.shape[0]
    if p.shape != (1864,) or xx.shape != (n, 16) or tt.shape != (n, 8):
        raise ValueError("params (1864,), x (n, 16), t (n, 8)")
    g = np.zeros(1864, np.float32)
    loss = C.c_double()
    sav = (C.c_double * 2)(*sa)
    _check(ctx.lib.stz_debug_mlp_grad(ctx._c, p.ctypes.data_as(C.c_void_p), xx.ctypes.data_as(C.c_void_p),
                                      tt.ctypes.data_as(C.c_void_p), n, s_in, s_t, huber_delta, int(qat), sav,
                                      g.ctypes.data_as(C.c_void_p), C.byref(loss)))
    return loss.value, g


def learned_infer(ctx: "Context", xq, record: bytes, tensor_cores: bool = True) -> np.ndarray:
    """The int8 network's output accumulators (n x 8 int32) for int8 input
    rows xq (n x 16), through stz_debug_learned_infer."""
    x = np.ascontiguousarray(xq, dtype=np.int8)
    if x.ndim != 2 or x.shape[1] != 16 or len(record) != 2112:
        raise ValueError("xq (n, 16) int8 and a 2112-byte model record")
    out = np.zeros((x.shape[0], 8), np.int32)
    rec = C.create_string_buffer(bytes(record), len(record))
    _check(ctx.lib.stz_debug_learned_infer(ctx._c, x.ctypes.data_as(C.c_void_p), x.shape[0], rec,
                                           int(tensor_cores), out.ctypes.data_as(C.c_void_p)))
    return out
