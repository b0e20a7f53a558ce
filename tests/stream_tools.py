"""Test helpers that rewrite a container's stream headers.

rewrite_plane_tables(stream, version, width) re-serialises every stream
header of a version-4 container with its plane table in another layout:
version 3 (u32 plane bit offsets inside the chunk) or version 4 with
`width`-byte plane bit counts (2 or 4). Header frames are stored raw after
the rewrite (a stored size equal to the raw size); payload frames are copied
unchanged. The directory layout is the one ContainerWriter::finish writes
(sc25-stz2_b200/csrc/host.cpp).

frame_sizes(stream) lists every frame's stored and raw size."""
import ctypes
import struct

import numpy as np

_zstd = ctypes.CDLL("libzstd.so.1")
_zstd.ZSTD_decompress.restype = ctypes.c_size_t


def _unzstd(src: bytes, raw: int) -> bytes:
    if len(src) == raw:
        return src
    buf = ctypes.create_string_buffer(raw)
    n = _zstd.ZSTD_decompress(buf, ctypes.c_size_t(raw), src, ctypes.c_size_t(len(src)))
    assert n == raw
    return buf.raw[:n]


def _plane_offsets(h: bytes, nch: int, C: int, elem: int, version: int):
    """(prefix bytes up to the marker table, offsets[nch][C])."""
    nu = struct.unpack_from("<I", h, 0)[0]
    p = 4 + 3 * nu + 8  # symbols, lengths, run_base, run_n
    nunp = struct.unpack_from("<Q", h, p)[0]
    p += 8 + nunp * elem + 4 * nch + 8 * (nch + 1)
    prefix = h[:p]
    if version >= 4:
        width = h[p]
        p += 1
        d = np.frombuffer(h, np.uint16 if width == 2 else np.uint32, nch * (C - 1), p).reshape(nch, C - 1)
        off = np.zeros((nch, C), np.uint64)
        off[:, 1:] = np.cumsum(d.astype(np.uint64), axis=1)
        p += d.nbytes
    else:
        off = np.frombuffer(h, np.uint32, nch * C, p).reshape(nch, C).astype(np.uint64)
        p += 4 * nch * C
    assert p == len(h)
    return prefix, off


def rewrite_plane_tables(b: bytes, version: int, width: int = 2) -> bytes:
    r = [8]

    def take(fmt):
        v = struct.unpack_from("<" + fmt, b, r[0])
        r[0] += struct.calcsize("<" + fmt)
        return v

    src_version = take("I")[0]
    assert src_version == 4
    dtype, _pred, _nx, _ny, _nz, K = take("6I")
    elem = 8 if dtype == 1 else 4
    take("3I")  # radius, chunk_high, chunk_low
    take("i")   # zstd level
    take("4d")  # eb, multipliers
    c0 = take("3I")
    r[0] += c0[0] * c0[1] * c0[2] * elem
    head = bytearray(b[:r[0]])
    struct.pack_into("<I", head, 8, version)
    levels = []
    for _ in range(K):
        dx, dy, dz, C = take("4I")
        (eb,) = take("d")
        (lf,) = take("I")
        model = b[r[0]:r[0] + 2112] if lf else b""
        r[0] += len(model)
        streams = []
        for _ in range(7):
            (L,) = take("I")
            hs, hr = take("2Q")
            ls = take(f"{L}Q")
            lr = take(f"{L}Q")
            streams.append((hs, hr, ls, lr))
        levels.append((dx, dy, dz, C, eb, lf, model, streams))
    pos = r[0]
    d = bytearray(head)
    frames = bytearray()
    for dx, dy, dz, C, eb, lf, model, streams in levels:
        d += struct.pack("<4I", dx, dy, dz, C) + struct.pack("<d", eb) + struct.pack("<I", lf) + model
        nch = (dx // C) * (dy // C) * (dz // C)
        for hs, hr, ls, lr in streams:
            h = _unzstd(b[pos:pos + hs], hr)
            pos += hs
            prefix, off = _plane_offsets(h, nch, C, elem, 4)
            if version >= 4:
                cnt = np.diff(off, axis=1)
                assert width == 4 or cnt.max(initial=0) < 65536
                table = bytes([width]) + cnt.astype(np.uint16 if width == 2 else np.uint32).tobytes()
            else:
                table = off.astype(np.uint32).tobytes()
            nh = prefix + table
            d += struct.pack("<I", len(ls)) + struct.pack("<2Q", len(nh), len(nh))
            d += struct.pack(f"<{len(ls)}Q", *ls) + struct.pack(f"<{len(lr)}Q", *lr)
            frames += nh + b[pos:pos + sum(ls)]
            pos += sum(ls)
    assert pos == len(b)
    return bytes(d + frames)


def frame_sizes(b: bytes):
    """[(level, block, kind, stored, raw)] for every frame of a version 2-4
    container; kind is "header" or "payload"."""
    r = [8]

    def take(fmt):
        v = struct.unpack_from("<" + fmt, b, r[0])
        r[0] += struct.calcsize("<" + fmt)
        return v

    version = take("I")[0]
    assert version >= 2
    dtype, _pred, _nx, _ny, _nz, K = take("6I")
    elem = 8 if dtype == 1 else 4
    take("3I")
    take("i")
    take("4d")
    c0 = take("3I")
    r[0] += c0[0] * c0[1] * c0[2] * elem
    out = []
    for k in range(1, K + 1):
        take("4I")
        take("d")
        (lf,) = take("I")
        r[0] += 2112 if lf else 0
        for blk in range(7):
            (L,) = take("I")
            hs, hr = take("2Q")
            ls = take(f"{L}Q")
            lr = take(f"{L}Q")
            out.append((k, blk, "header", hs, hr))
            out += [(k, blk, "payload", a, c) for a, c in zip(ls, lr)]
    return out
