"""ctypes wrapper of liboracle.so, the CPU float64 oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py, never by the radix_b200 package.
"""
import ctypes
import os
import subprocess

import numpy as np

from radix_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


class orc_grads_in(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in ("mean2d", "conic", "depth", "opacity", "rgb")]


class orc_grads_out(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in ("centers", "log_scales", "quats", "opacities", "colors")]


class orc_splat(ctypes.Structure):
    _fields_ = [("center", ctypes.c_double * 3), ("scales", ctypes.c_double * 3), ("quat", ctypes.c_double * 4),
                ("opacity", ctypes.c_double), ("rgb", ctypes.c_double * 3), ("sh", ctypes.c_double * 72),
                ("sh_degree", ctypes.c_int), ("cov", ctypes.c_double * 6), ("has_cov", ctypes.c_int)]


class orc_outputs(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in
                ("mean2d", "conic", "depth", "opacity", "rgb", "radii", "words", "keys", "distance", "visible")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32, f64, vp, i = ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p, ctypes.c_int
        sigs = {
            "orc_invalid_key": (u32, [i]),
            "orc_valid_max": (u32, [i]),
            "orc_sort_key": (u32, [f64, i]),
            "orc_sort_key_f32": (u32, [ctypes.c_float, i]),
            "orc_sort_keys": (None, [vp, ctypes.c_uint64, i, vp]),
            "orc_sort": (i, [vp, ctypes.c_uint64, i, vp, ctypes.c_uint64, vp]),
            "orc_decode_half": (f64, [u32]),
            "orc_encode_half": (u32, [f64]),
            "orc_decode_ext_rgb": (None, [u32, vp]),
            "orc_encode_ext_rgb": (u32, [vp]),
            "orc_decode_oct": (None, [u32, i, vp]),
            "orc_encode_oct": (u32, [vp, i]),
            "orc_decode_quat_oct32": (None, [u32, vp]),
            "orc_encode_quat_oct32": (u32, [vp]),
            "orc_sh_basis": (None, [vp, vp]),
            "orc_sh_evaluate": (None, [vp, vp, i, vp]),
            "orc_project": (i, [ctypes.POINTER(_abi.rdx_object), i, ctypes.POINTER(_abi.rdx_camera),
                                ctypes.POINTER(_abi.rdx_params), i, i, i, ctypes.POINTER(orc_outputs)]),
            "orc_project_rays": (i, [ctypes.POINTER(_abi.rdx_object), i, ctypes.POINTER(_abi.rdx_camera),
                                     ctypes.POINTER(_abi.rdx_params), i, i, i, i, vp, vp]),
            "orc_encode_ext_table": (i, [ctypes.POINTER(_abi.rdx_table), vp, vp, vp]),
            "orc_sh_basis_grad": (None, [vp, vp]),
            "orc_ply_decode": (i, [vp, ctypes.c_uint64, i, vp, vp, vp, vp, vp, vp, vp, vp]),
            "orc_spz_decode": (i, [i, ctypes.c_uint64, i, i, vp, vp, vp, vp, vp, vp, i, vp, vp, vp, vp, vp]),
            "orc_load_splat": (None, [ctypes.POINTER(_abi.rdx_table), ctypes.c_uint64, ctypes.POINTER(orc_splat)]),
            "orc_encode_packed_table": (i, [ctypes.POINTER(_abi.rdx_table), vp, vp]),
            "orc_encode_cov_table": (i, [ctypes.POINTER(_abi.rdx_table), vp, vp]),
            "orc_sh_words": (i, [i, i]),
            "orc_encode_sh": (i, [ctypes.POINTER(_abi.rdx_table), i, vp, i]),
            "orc_decode_quat_oct": (None, [u32, i, i, vp]),
            "orc_encode_quat_oct": (u32, [vp, i, i]),
            "orc_project_backward": (i, [ctypes.POINTER(_abi.rdx_object), i, ctypes.POINTER(_abi.rdx_camera),
                                         ctypes.POINTER(_abi.rdx_params), ctypes.POINTER(orc_grads_in),
                                         ctypes.POINTER(orc_grads_out), i]),
            "orc_params_default": (None, [ctypes.POINTER(_abi.rdx_params)]),
            "orc_encode_depth20": (u32, [f64]),
            "orc_encode_angle12": (u32, [f64]),
            "orc_mat4_mul": (None, [vp, vp, vp]),
            "orc_mat4_invert": (i, [vp, vp]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data


def sort_key(distance, bits):
    return lib().orc_sort_key(float(distance), bits)


def sort_key_f32(distance, bits):
    return lib().orc_sort_key_f32(float(np.float32(distance)), bits)


def sort_keys(distances, bits):
    d = np.ascontiguousarray(distances, dtype=np.float64)
    out = np.empty(d.size, dtype=np.uint32)
    lib().orc_sort_keys(_p(d), d.size, bits, _p(out))
    return out


def sort(keys, count=None, bits=32, ordering_len=None):
    """SortKeys.sort: (ordering, visible); ValueError when ordering_len < count."""
    k = np.ascontiguousarray(keys, dtype=np.uint32)
    count = k.size if count is None else count
    ordering_len = max(1, -(-count // 4096)) * 4096 if ordering_len is None else ordering_len
    ordering = np.zeros(max(ordering_len, 1), dtype=np.uint32)
    visible = ctypes.c_uint32(0)
    if lib().orc_sort(_p(k), count, bits, _p(ordering), ordering_len, ctypes.addressof(visible)) != 0:
        raise ValueError(f"SortKeys.sort: ordering holds {ordering_len} of {count} indices")
    return ordering[:ordering_len], visible.value


def decode_half(h):
    return lib().orc_decode_half(int(h))


def encode_half(f):
    return lib().orc_encode_half(float(f))


def decode_ext_rgb(w):
    out = np.zeros(3)
    lib().orc_decode_ext_rgb(int(w), _p(out))
    return out


def encode_ext_rgb(rgb):
    a = np.ascontiguousarray(rgb, dtype=np.float64)
    return lib().orc_encode_ext_rgb(_p(a))


def decode_quat_oct32(code):
    out = np.zeros(4)
    lib().orc_decode_quat_oct32(int(code), _p(out))
    return out


def encode_quat_oct32(q):
    a = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_encode_quat_oct32(_p(a))


def sh_basis(d):
    a = np.ascontiguousarray(d, dtype=np.float64)
    out = np.zeros(24)
    lib().orc_sh_basis(_p(a), _p(out))
    return out


def sh_evaluate(coeffs, d, degree):
    c = np.zeros(72)
    flat = np.asarray(coeffs, dtype=np.float64).reshape(-1)
    c[:flat.size] = flat
    a = np.ascontiguousarray(d, dtype=np.float64)
    out = np.zeros(3)
    lib().orc_sh_evaluate(_p(c), _p(a), int(degree), _p(out))
    return out


def params_default():
    p = _abi.rdx_params()
    lib().orc_params_default(ctypes.byref(p))
    return p


def project(objects, camera, params=None, sort_bits=24, cull_keys=False, threads=0):
    """The float64 projection of radix_b200.SplatObject's (numpy tables) for a
    radix_b200.Camera: a dict of float64 / uint32 arrays."""
    import radix_b200 as rb
    params = params or rb.SplatParams()
    n = sum(o.count for o in objects)
    E = len(camera.eyes)
    out = {
        "mean2d": np.zeros((E, n, 2)), "conic": np.zeros((E, n, 3)), "depth": np.zeros((E, n)),
        "opacity": np.zeros((E, n)), "rgb": np.zeros((E, n, 3)), "radii": np.zeros((E, n, 3)),
        "words": np.zeros((n, 4 * E), dtype=np.uint32), "keys": np.zeros(n, dtype=np.uint32),
        "distance": np.zeros(n), "visible": np.zeros((E, n), dtype=np.uint8),
    }
    o = orc_outputs(**{k: _p(v) for k, v in out.items()})
    objs, keep = rb._c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    st = lib().orc_project(objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), sort_bits,
                           1 if cull_keys else 0, threads, ctypes.byref(o))
    del keep
    if st != 0:
        raise ValueError("orc_project failed")
    return out


RAY_METHODS = {"3dgut": 1, "htgs": 2, "raygs": 3}
RAY_WORDS = {"3dgut": (6, 2), "htgs": (6, 2), "raygs": (4, 3)}  # head words, words per eye


def project_rays(objects, camera, method, params=None, sort_bits=24, cull_keys=False, threads=0):
    """The float64 words and keys of a ray projection method ("3dgut", "htgs",
    "raygs"): {"words": uint32 [n][H + E * W], "keys": uint32 [n]}."""
    import radix_b200 as rb
    params = params or rb.SplatParams()
    n = sum(o.count for o in objects)
    head, per_eye = RAY_WORDS[method]
    words = np.zeros((n, head + len(camera.eyes) * per_eye), dtype=np.uint32)
    keys = np.zeros(n, dtype=np.uint32)
    objs, keep = rb._c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    st = lib().orc_project_rays(objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), RAY_METHODS[method],
                                sort_bits, 1 if cull_keys else 0, threads, _p(words), _p(keys))
    del keep
    if st != 0:
        raise ValueError("orc_project_rays failed (%d)" % st)
    return {"words": words, "keys": keys}


def encode_ext(raw):
    """(ext_a, ext_b, [ext_sh channels]) of a numpy raw table dict (float32 colours)."""
    import radix_b200 as rb
    t = rb.Table.from_dict(raw)
    n = t.count
    deg = raw["sh_degree"]
    texels = ((deg + 1) ** 2 - 1 + 3) // 4
    a = np.zeros((n, 4), dtype=np.uint32)
    b = np.zeros((n, 4), dtype=np.uint32)
    sh = [np.zeros((n, 4), dtype=np.uint32) for _ in range(texels)]
    ptrs = (ctypes.c_void_p * 6)(*([_p(c) for c in sh] + [None] * (6 - texels)))
    if lib().orc_encode_ext_table(ctypes.byref(t.c), _p(a), _p(b), ptrs) != 0:
        raise ValueError("orc_encode_ext_table failed")
    return a, b, sh


def project_backward(objects, camera, upstream, params=None, threads=0):
    """float64 gradient of the projection's mean2d / conic / depth / opacity /
    rgb (upstream: dict of arrays shaped as project()'s outputs, missing =
    zero) with respect to the raw tables' rows: dict of centers [n][3],
    log_scales [n][3], quats [n][4], opacities [n] and colors [n][75]."""
    import radix_b200 as rb
    params = params or rb.SplatParams()
    n = sum(o.count for o in objects)
    ups = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in upstream.items() if v is not None}
    gin = orc_grads_in(**{k: _p(v) for k, v in ups.items()})
    out = {"centers": np.zeros((n, 3)), "log_scales": np.zeros((n, 3)), "quats": np.zeros((n, 4)),
           "opacities": np.zeros(n), "colors": np.zeros((n, 75))}
    gout = orc_grads_out(**{k: _p(v) for k, v in out.items()})
    objs, keep = rb._c_objects(objects)
    cam = camera.to_c(_abi)
    prm = params.to_c()
    st = lib().orc_project_backward(objs, len(objects), ctypes.byref(cam), ctypes.byref(prm), ctypes.byref(gin),
                                    ctypes.byref(gout), threads)
    del keep, ups
    if st != 0:
        raise ValueError("orc_project_backward failed (ext tables have no gradient)")
    return out


def sh_basis_grad(d):
    out = np.zeros((24, 3))
    lib().orc_sh_basis_grad(_p(np.ascontiguousarray(d, dtype=np.float64)), _p(out))
    return out


def encode_packed(raw, encoding=(0.0, 1.0, -12.0, 9.0)):
    """packedCodec.encode of a numpy raw table dict: [n][4] uint32."""
    import radix_b200 as rb
    t = rb.Table.from_dict(raw)
    out = np.zeros((t.count, 4), dtype=np.uint32)
    enc = np.asarray(encoding, dtype=np.float32)
    if lib().orc_encode_packed_table(ctypes.byref(t.c), _p(enc), _p(out)) != 0:
        raise ValueError("orc_encode_packed_table failed")
    return out


def encode_cov(raw):
    """storeCovFields of a numpy raw table dict: (covA, covB), [n][4] uint32 each."""
    import radix_b200 as rb
    t = rb.Table.from_dict(raw)
    a = np.zeros((t.count, 4), dtype=np.uint32)
    b = np.zeros((t.count, 4), dtype=np.uint32)
    if lib().orc_encode_cov_table(ctypes.byref(t.c), _p(a), _p(b)) != 0:
        raise ValueError("orc_encode_cov_table failed")
    return a, b


def encode_sh(raw, codec):
    """A raw table's SH coefficients as codec words ("ext" / "packed"):
    [n][texels * 4] uint32, zero padded to whole texels."""
    import radix_b200 as rb
    t = rb.Table.from_dict(raw)
    c = _abi.RDX_SH_PACKED if codec == "packed" else _abi.RDX_SH_EXT
    words = lib().orc_sh_words(c, raw["sh_degree"])
    stride = (words + 3) // 4 * 4
    out = np.zeros((t.count, max(stride, 4)), dtype=np.uint32)
    if lib().orc_encode_sh(ctypes.byref(t.c), c, _p(out), out.shape[1]) != 0:
        raise ValueError("orc_encode_sh failed")
    return out[:, :stride] if stride else out[:, :0]


def sh_channels(words):
    """Codec words [n][4 * texels] as per-splat texel channels [n][4] each."""
    return [np.ascontiguousarray(words[:, 4 * k:4 * k + 4]) for k in range(words.shape[1] // 4)]


def sh_palette(words, stride):
    """Entries' codec words [size][4 * texels] as an ShPalette's shEntries:
    [size * stride][4], each entry `stride` texels (the tail zero)."""
    size, w = words.shape
    out = np.zeros((size, stride, 4), dtype=np.uint32)
    out[:, :w // 4, :] = words.reshape(size, w // 4, 4)
    return out.reshape(size * stride, 4)


def load_splat(table, i):
    """orc_load_splat of row i of a radix_b200.Table (numpy columns): a dict."""
    sp = orc_splat()
    lib().orc_load_splat(ctypes.byref(table.c), i, ctypes.byref(sp))
    k = ((sp.sh_degree + 1) ** 2 - 1) * 3
    return {"center": np.array(sp.center[:]), "scales": np.array(sp.scales[:]), "quat": np.array(sp.quat[:]),
            "opacity": sp.opacity, "rgb": np.array(sp.rgb[:]), "sh": np.array(sp.sh[:k]),
            "cov": np.array(sp.cov[:]) if sp.has_cov else None}


def ply_decode(data, sh_degree=-1):
    """orc_ply_decode of PLY bytes: a dict of float64 raw-table columns plus
    count, sh_degree (the file's) and kind (0 standard, 1 points, 2 compressed)."""
    buf = np.frombuffer(bytes(data), dtype=np.uint8)
    n = ctypes.c_uint64(0)
    deg = ctypes.c_int(0)
    kind = ctypes.c_int(0)
    if lib().orc_ply_decode(_p(buf), buf.size, -1, None, None, None, None, None, ctypes.byref(n), ctypes.byref(deg),
                            ctypes.byref(kind)) != 0:
        raise ValueError("orc_ply_decode: malformed PLY")
    d = deg.value if sh_degree < 0 else sh_degree
    count = n.value
    row = ((d + 1) ** 2) * 3
    out = {"centers": np.zeros((count, 3)), "log_scales": np.zeros((count, 3)), "quats": np.zeros((count, 4)),
           "opacities": np.zeros(count), "colors": np.zeros((count, row // 3, 3))}
    if lib().orc_ply_decode(_p(buf), buf.size, d, _p(out["centers"]), _p(out["log_scales"]), _p(out["quats"]),
                            _p(out["opacities"]), _p(out["colors"]), ctypes.byref(n), ctypes.byref(deg),
                            ctypes.byref(kind)) != 0:
        raise ValueError("orc_ply_decode: malformed PLY")
    out.update(count=count, sh_degree=deg.value, kind=kind.value, degree=d)
    return out


# ---- SPZ (src/core/spz.ts): the two containers unpacked here, the splats decoded by orc_spz_decode ----

SPZ_MAGIC = 0x5053474E  # "NGSP" little-endian
SPZ_SH_VECTORS = {0: 0, 1: 3, 2: 8, 3: 15, 4: 24}


def zstd_lib():
    """libzstd (the system's shared library), for SPZ 4's streams; None when absent."""
    try:
        z = ctypes.CDLL("libzstd.so.1")
    except OSError:
        return None
    z.ZSTD_decompress.restype = ctypes.c_size_t
    z.ZSTD_decompress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
    z.ZSTD_isError.restype = ctypes.c_uint
    z.ZSTD_isError.argtypes = [ctypes.c_size_t]
    z.ZSTD_compress.restype = ctypes.c_size_t
    z.ZSTD_compress.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    z.ZSTD_compressBound.restype = ctypes.c_size_t
    z.ZSTD_compressBound.argtypes = [ctypes.c_size_t]
    return z


def _le32(b, at):
    return int.from_bytes(b[at:at + 4], "little")


def _spz_check(version, degree, latest):
    if version < 1 or version > latest or degree not in SPZ_SH_VECTORS:
        raise ValueError(f"Unsupported SPZ version {version} or SH degree {degree}")


def spz_unpack(data):
    """unpackSpz (src/core/spz.ts:141-263): the header and byte columns of an
    SPZ file in either container, with the reference's error texts."""
    import zlib
    raw = bytes(data)
    if len(raw) >= 4 and _le32(raw, 0) == SPZ_MAGIC:
        if len(raw) < 32:
            raise ValueError("SPZ file ended unexpectedly")
        version, count = _le32(raw, 4), _le32(raw, 8)
        degree, fb, flags, nstreams = raw[12], raw[13], raw[14], raw[15]
        toc_at = _le32(raw, 16)
        if version != 4:
            raise ValueError(f"Unsupported SPZ version {version} in the NGSP container")
        _spz_check(version, degree, 4)
        if count > 0x7FFFFFFF:
            raise ValueError(f"Invalid SPZ point count {count}")
        if toc_at < 32:
            raise ValueError("SPZ 4 table of contents inside the header")
        sizes = [count * b for b in (9, 1, 3, 3, 4, SPZ_SH_VECTORS[degree] * 3)]
        present = [k for k, size in enumerate(sizes) if size > 0]
        if nstreams != len(present):
            raise ValueError(f"SPZ 4 file with {nstreams} streams, {len(present)} expected")
        if len(raw) < toc_at + nstreams * 16:
            raise ValueError("SPZ file ended unexpectedly")
        total = toc_at + nstreams * 16
        comp = []
        for k in range(nstreams):
            low, high, size_low, size_high = (_le32(raw, toc_at + k * 16 + a) for a in (0, 4, 8, 12))
            if high >= 1 << 21 or size_high != 0 or size_low != sizes[present[k]]:
                raise ValueError(f"SPZ 4 stream {k} sizes don't match its header")
            comp.append(high * 2 ** 32 + low)
            total += comp[-1]
        if count * 9 > total * 1024:
            raise ValueError(f"Invalid SPZ point count {count} for {total} bytes")
        z = zstd_lib()
        if z is None:
            raise ValueError("SPZ 4 needs libzstd")
        cols = [b""] * 6
        at = toc_at + nstreams * 16
        for k in range(nstreams):
            if at + comp[k] > len(raw):
                raise ValueError("SPZ file ended unexpectedly")
            src = np.frombuffer(raw[at:at + comp[k]], dtype=np.uint8)
            dst = np.zeros(max(sizes[present[k]], 1), dtype=np.uint8)
            got = z.ZSTD_decompress(_p(dst), sizes[present[k]], _p(src), comp[k])
            if z.ZSTD_isError(got) or got != sizes[present[k]]:
                raise ValueError(f"SPZ 4 stream {k} does not decompress to its size")
            cols[present[k]] = dst[:sizes[present[k]]].tobytes()
            at += comp[k]
        if at != len(raw):
            raise ValueError("SPZ 4 file has bytes after its last stream")
        return {"container": "ngsp", "version": version, "count": count, "sh_degree": degree,
                "fractional_bits": fb, "flags": flags, "centers": cols[0], "alphas": cols[1], "colors": cols[2],
                "scales": cols[3], "rotations": cols[4], "sh": cols[5]}
    if raw[:2] != b"\x1f\x8b":
        raise ValueError("Invalid SPZ file")
    d = zlib.decompressobj(wbits=31)
    payload = d.decompress(raw)
    while d.eof and d.unused_data:  # concatenated gzip members
        rest = d.unused_data
        d = zlib.decompressobj(wbits=31)
        payload += d.decompress(rest)
    if len(payload) < 16:
        raise ValueError("SPZ file ended unexpectedly")
    if _le32(payload, 0) != SPZ_MAGIC:
        raise ValueError("Invalid SPZ file")
    version, count = _le32(payload, 4), _le32(payload, 8)
    degree, fb, flags = payload[12], payload[13], payload[14]
    _spz_check(version, degree, 4)
    sizes = [count * (6 if version == 1 else 9), count, count * 3, count * 3, count * (4 if version >= 3 else 3),
             count * SPZ_SH_VECTORS[degree] * 3]
    at, cols = 16, []
    for size in sizes:
        if at + size > len(payload):
            raise ValueError("SPZ file ended unexpectedly")
        cols.append(payload[at:at + size])
        at += size
    return {"container": "gzip", "version": version, "count": count, "sh_degree": degree, "fractional_bits": fb,
            "flags": flags, "centers": cols[0], "alphas": cols[1], "colors": cols[2], "scales": cols[3],
            "rotations": cols[4], "sh": cols[5]}


def spz_decode(data, sh_degree=-1):
    """SpzFile.read's splats (src/core/spz.ts:265-348) as float64 raw-table
    columns (orc_spz_decode), plus the header fields."""
    u = spz_unpack(data)
    deg = u["sh_degree"] if sh_degree < 0 else sh_degree
    if deg > u["sh_degree"]:
        raise ValueError(f"the file has SH degree {u['sh_degree']}, not {deg}")
    n = u["count"]
    out = {"centers": np.zeros((n, 3)), "log_scales": np.zeros((n, 3)), "quats": np.zeros((n, 4)),
           "opacities": np.zeros(n), "colors": np.zeros((n, (deg + 1) ** 2, 3))}
    cols = [np.frombuffer(u[k], dtype=np.uint8) if len(u[k]) else np.zeros(1, dtype=np.uint8)
            for k in ("centers", "alphas", "colors", "scales", "rotations", "sh")]
    if lib().orc_spz_decode(u["version"], n, u["sh_degree"], u["fractional_bits"], *(_p(c) for c in cols), deg,
                            _p(out["centers"]), _p(out["log_scales"]), _p(out["quats"]), _p(out["opacities"]),
                            _p(out["colors"])) != 0:
        raise ValueError("orc_spz_decode: bad arguments")
    out.update({k: u[k] for k in ("container", "version", "count", "sh_degree", "fractional_bits", "flags")})
    out["degree"] = deg
    return out


# ---- RDX files (src/core/rdx.ts:62-205): containers, byte-transposed gzip payloads ----

RDX_HEADER_MAGIC = 0x48584452  # "RDXH"
RDX_CHUNK_MAGIC = 0x43584452   # "RDXC"
_RDX_SCALARS = {"uint8": 1, "sint8": 1, "unorm8": 1, "snorm8": 1, "uint16": 2, "sint16": 2, "float16": 2,
                "uint32": 4, "sint32": 4, "float32": 4}


def _rdx_container(raw, at, magic):
    """decodeContainer: (meta, [payload bytes], byte length) of the piece at `at`."""
    import json
    if len(raw) - at < 16 or _le32(raw, at) != magic:
        raise ValueError("Not an RDX piece of the expected type")
    meta_len, count = _le32(raw, at + 4), _le32(raw, at + 8)
    meta = json.loads(raw[at + 16:at + 16 + meta_len].decode())
    sizes_at = at + 16 + (meta_len + 15) // 16 * 16
    off = sizes_at + (count * 4 + 15) // 16 * 16
    payloads = []
    for i in range(count):
        size = _le32(raw, sizes_at + 4 * i)
        if off + size > len(raw):
            raise ValueError("RDX file ended unexpectedly")
        payloads.append(raw[off:off + size])
        off += (size + 15) // 16 * 16
    return meta, payloads, off - at


def rdxfile_read(data):
    """RdxFile.read of a whole file: (header, {bundle: {label: uint8 array [count, element bytes]}})."""
    import zlib
    raw = bytes(data)
    header, _, length = _rdx_container(raw, 0, RDX_HEADER_MAGIC)
    if header.get("version") != 1:
        raise ValueError(f"RDX version {header.get('version')} is not 1")
    count = header["count"]
    chans = []
    for name, b in header["bundles"].items():
        for label, fmt in b["def"]["channels"].items():
            scalar, _, comps = fmt.partition("x")
            chans.append((name, label, _RDX_SCALARS[scalar] * (int(comps) if comps else 1)))
    out = {name: {} for name, _, _ in chans}
    for name, label, eb in chans:
        out[name][label] = np.zeros((count, eb), dtype=np.uint8)
    at = length
    for size in header["chunks"]:
        meta, payloads, _ = _rdx_container(raw, at, RDX_CHUNK_MAGIC)
        start, n = meta["start"], meta["count"]
        for (name, label, eb), p in zip(chans, payloads):
            t = np.frombuffer(zlib.decompress(p, 31), dtype=np.uint8)
            if t.size != n * eb:
                raise ValueError(f"Chunk at {start}: {name}.{label} holds {t.size} bytes, expected {n * eb}")
            out[name][label][start:start + n] = t.reshape(eb, n).T
        at += size
    return header, out
