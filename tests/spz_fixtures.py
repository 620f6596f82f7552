"""Writers of SPZ test files from synthetic raw tables, restating the
quantisation of SpzFile.write (src/core/spz.ts:388-560): 24-bit fixed-point
centres (halves in version 1), alpha and colour bytes, log-scale bytes
(ln s + 10) * 16, rotations as smallest three (versions 3 and 4) or 3 bytes of
x y z with w >= 0 (versions 1 and 2), SH bytes b * 128 + 128; in gzip (one
member or several) or in SPZ 4's NGSP container (one zstd stream per
non-empty column, a table of contents, optional extension records)."""
import ctypes
import gzip
import math
import struct

import numpy as np

SPZ_MAGIC = 0x5053474E  # "NGSP" little-endian
SH_C0 = 0.28209479177387814
COLOR_SCALE = SH_C0 / 0.15
SH_VECTORS = {0: 0, 1: 3, 2: 8, 3: 15, 4: 24}


def zstd():
    """libzstd through ctypes (the system's shared library), or None."""
    try:
        z = ctypes.CDLL("libzstd.so.1")
    except OSError:
        return None
    z.ZSTD_compress.restype = ctypes.c_size_t
    z.ZSTD_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    z.ZSTD_compressBound.restype = ctypes.c_size_t
    z.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
    z.ZSTD_isError.restype = ctypes.c_uint
    z.ZSTD_isError.argtypes = [ctypes.c_size_t]
    return z


def _byte(x):
    """Math.round(clamp(x, 0, 255)): halves round up."""
    return np.floor(np.clip(np.asarray(x, dtype=np.float64), 0.0, 255.0) + 0.5).astype(np.uint8)


def _smallest_three(q):
    n = q / np.linalg.norm(q, axis=1, keepdims=True)
    largest = np.argmax(np.abs(n), axis=1)
    negate = n[np.arange(len(n)), largest] < 0
    packed = largest.astype(np.uint64)
    for i in range(4):
        keep = largest != i
        sign = ((n[:, i] < 0) ^ negate).astype(np.uint64)
        mag = np.clip(np.floor(511.0 * np.abs(n[:, i]) / math.sqrt(0.5) + 0.5), 0, 511).astype(np.uint64)
        packed = np.where(keep, (packed << np.uint64(10)) | (sign << np.uint64(9)) | mag, packed)
    return (packed & np.uint64(0xFFFFFFFF)).astype(np.uint32)


def columns(d, version=3, fractional_bits=12, sh_degree=None):
    """The byte columns of a raw table dict: centers, alphas, colors, scales, rotations, sh."""
    n = d["centers"].shape[0]
    deg = d.get("sh_degree", 0) if sh_degree is None else sh_degree
    c = d["centers"].astype(np.float64)
    if version == 1:
        centers = c.astype("<f2").tobytes()  # float64 to half, ties to even
    else:
        code = np.clip(np.floor(c * (1 << fractional_bits) + 0.5), -0x7FFFFF, 0x7FFFFF).astype(np.int64) & 0xFFFFFF
        centers = np.stack([code & 0xFF, (code >> 8) & 0xFF, (code >> 16) & 0xFF], axis=-1).astype(np.uint8).tobytes()
    alphas = _byte(d["opacities"].astype(np.float64) * 255).tobytes()
    rgb = d["colors"][:, 0, :].astype(np.float64)
    colors = _byte(((rgb - 0.5) / COLOR_SCALE + 0.5) * 255).tobytes()
    scales = _byte((d["log_scales"].astype(np.float64) + 10) * 16).tobytes()
    q = d["quats"].astype(np.float64)
    if version >= 3:
        rotations = _smallest_three(q).astype("<u4").tobytes()
    else:
        n4 = q / np.linalg.norm(q, axis=1, keepdims=True)
        sign = np.where(n4[:, 3] < 0, -1.0, 1.0)[:, None]
        rotations = _byte((n4[:, :3] * sign + 1) * 127.5).tobytes()
    k = SH_VECTORS[deg]
    sh = _byte(d["colors"][:, 1:1 + k, :].astype(np.float64) * 128 + 128).tobytes() if k else b""
    return [centers, alphas, colors, scales, rotations, sh], deg


def gzip_spz(d, version=3, fractional_bits=12, sh_degree=None, members=1, flags=0x01, trailer=b"", level=9):
    """A gzip SPZ (versions 1 to 4: 4 is version 3's layout) of a raw table
    dict, at gzip compression `level`."""
    cols, deg = columns(d, version, fractional_bits, sh_degree)
    n = d["centers"].shape[0]
    head = struct.pack("<IIIBBBB", SPZ_MAGIC, version, n, deg, fractional_bits, flags, 0)
    body = head + b"".join(cols) + trailer
    if members == 1:
        return gzip.compress(body, compresslevel=level, mtime=0)
    cut = len(body) // members
    parts = [body[i * cut:(i + 1) * cut if i < members - 1 else len(body)] for i in range(members)]
    return b"".join(gzip.compress(p, compresslevel=level, mtime=0) for p in parts)


def ngsp_spz(d, fractional_bits=12, sh_degree=None, records=b"", flags=0x01, level=3):
    """An SPZ 4 file (NGSP container) of a raw table dict."""
    z = zstd()
    cols, deg = columns(d, 3, fractional_bits, sh_degree)
    n = d["centers"].shape[0]
    streams, sizes = [], []
    for col in cols:
        if not col:
            continue
        src = np.frombuffer(col, dtype=np.uint8)
        dst = np.zeros(z.ZSTD_compressBound(len(col)), dtype=np.uint8)
        got = z.ZSTD_compress(dst.ctypes.data, dst.size, src.ctypes.data, src.size, level)
        assert not z.ZSTD_isError(got)
        streams.append(dst[:got].tobytes())
        sizes.append(len(col))
    toc_at = 32 + len(records)
    head = struct.pack("<IIIBBBBI", SPZ_MAGIC, 4, n, deg, fractional_bits, flags | (0x02 if records else 0),
                       len(streams), toc_at) + b"\0" * 12
    toc = b"".join(struct.pack("<IIII", len(s) & 0xFFFFFFFF, len(s) >> 32, size, 0) for s, size in zip(streams, sizes))
    return head + records + toc + b"".join(streams)


def record(kind, payload):
    return struct.pack("<II", kind, len(payload)) + payload
