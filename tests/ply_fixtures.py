"""Writers of PLY test files from synthetic tables: standard 3DGS (writePly's
property order, src/core/ply.ts:290-359), RGB point clouds, and SuperSplat
compressed files (chunks of 256 with per-chunk ranges, 11/10/11-bit
positions and log scales, smallest-three 10-bit rotations, 8-bit colours and
opacity, an optional uchar sh element), in either byte order."""
import math

import numpy as np

SH_C0 = 0.28209479177387814


def _header(elements, little=True, comment="radix_b200 test fixture"):
    lines = ["ply", f"format binary_{'little' if little else 'big'}_endian 1.0", f"comment {comment}"]
    for name, count, props in elements:
        lines.append(f"element {name} {count}")
        lines += [f"property {t} {p}" for p, t in props]
    lines.append("end_header")
    return ("\n".join(lines) + "\n").encode()


def _records(columns, little=True):
    """Structured records of (name, numpy dtype char, values [n]) columns."""
    order = "<" if little else ">"
    dt = np.dtype([(name, order + ch) for name, ch, _ in columns])
    rec = np.zeros(len(columns[0][2]), dtype=dt)
    for name, _, vals in columns:
        rec[name] = vals
    return rec.tobytes()


def standard_ply(d, little=True, extra_uchar=False, comment="radix_b200 test fixture", extra_doubles=0):
    """A standard 3DGS PLY of a raw table dict (float properties; opacity as a
    logit); the comment's length sets where the records start, and
    extra_doubles unread double properties lengthen each record."""
    n = d["centers"].shape[0]
    deg = d["sh_degree"]
    k = (deg + 1) ** 2 - 1
    cols = [("x", "f4", d["centers"][:, 0]), ("y", "f4", d["centers"][:, 1]), ("z", "f4", d["centers"][:, 2])]
    if extra_uchar:  # an odd-sized property: records no longer 4-byte aligned
        cols.append(("flag", "u1", np.arange(n) % 7))
    cols += [(f"f_dc_{c}", "f4", (d["colors"][:, 0, c].astype(np.float64) - 0.5) / SH_C0) for c in range(3)]
    # f_rest channel-major: f_rest_{c * k + j} is coefficient j's channel c
    cols += [(f"f_rest_{c * k + j}", "f4", d["colors"][:, 1 + j, c]) for c in range(3) for j in range(k)]
    op = np.clip(d["opacities"].astype(np.float64), 1e-6, 1 - 1e-6)
    cols.append(("opacity", "f4", np.log(op / (1 - op))))
    cols += [(f"scale_{c}", "f4", d["log_scales"][:, c]) for c in range(3)]
    q = d["quats"]
    cols += [("rot_0", "f4", q[:, 3]), ("rot_1", "f4", q[:, 0]), ("rot_2", "f4", q[:, 1]), ("rot_3", "f4", q[:, 2])]
    cols += [(f"extra_{e}", "f8", np.full(n, e + 0.5)) for e in range(extra_doubles)]
    types = {"f4": "float", "u1": "uchar", "f8": "double"}
    head = _header([("vertex", n, [(name, types[ch]) for name, ch, _ in cols])], little, comment)
    return head + _records(cols, little)


def point_cloud_ply(n, seed=0, alpha=True, little=True):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(size=(n, 3)).astype(np.float32)
    rgb = rng.integers(0, 256, size=(n, 3))
    cols = [("x", "f4", xyz[:, 0]), ("y", "f4", xyz[:, 1]), ("z", "f4", xyz[:, 2]),
            ("red", "u1", rgb[:, 0]), ("green", "u1", rgb[:, 1]), ("blue", "u1", rgb[:, 2])]
    if alpha:
        cols.append(("alpha", "u2", rng.integers(0, 65536, size=n)))
    types = {"f4": "float", "u1": "uchar", "u2": "ushort"}
    return _header([("vertex", n, [(name, types[ch]) for name, ch, _ in cols])], little) + _records(cols, little)


def compressed_ply(d, little=True, sh=True, color_ranges=True):
    """A compressed PLY of a raw table dict (table order)."""
    n = d["centers"].shape[0]
    chunks = (n + 255) // 256
    c = d["centers"].astype(np.float64)
    ls = np.clip(d["log_scales"].astype(np.float64), -20, 20)
    rgb = d["colors"][:, 0].astype(np.float64)
    q = d["quats"].astype(np.float64)
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    pad = chunks * 256 - n

    def ranges(x):
        xp = np.concatenate([x, np.repeat(x[-1:], pad, axis=0)]).reshape(chunks, 256, -1)
        return xp.min(axis=1), xp.max(axis=1)

    cmin, cmax = ranges(c)
    smin, smax = ranges(ls)
    rmin, rmax = ranges(rgb) if color_ranges else (np.zeros((chunks, 3)), np.ones((chunks, 3)))
    ci = np.arange(n) // 256

    def quant(x, lo, hi, bits):
        m = (1 << bits) - 1
        t = np.where(hi > lo, (x - lo) / np.where(hi > lo, hi - lo, 1), 0)
        return np.clip(np.round(t * m), 0, m).astype(np.uint64)

    pos = (quant(c[:, 0], cmin[ci, 0], cmax[ci, 0], 11) << 21) | (quant(c[:, 1], cmin[ci, 1], cmax[ci, 1], 10) << 11) \
        | quant(c[:, 2], cmin[ci, 2], cmax[ci, 2], 11)
    scl = (quant(ls[:, 0], smin[ci, 0], smax[ci, 0], 11) << 21) | (quant(ls[:, 1], smin[ci, 1], smax[ci, 1], 10) << 11) \
        | quant(ls[:, 2], smin[ci, 2], smax[ci, 2], 11)
    col = (quant(rgb[:, 0], rmin[ci, 0], rmax[ci, 0], 8) << 24) | (quant(rgb[:, 1], rmin[ci, 1], rmax[ci, 1], 8) << 16) \
        | (quant(rgb[:, 2], rmin[ci, 2], rmax[ci, 2], 8) << 8) \
        | np.clip(np.round(d["opacities"].astype(np.float64) * 255), 0, 255).astype(np.uint64)
    # smallest three of (w, x, y, z), the largest's index in the top 2 bits
    wxyz = np.stack([q[:, 3], q[:, 0], q[:, 1], q[:, 2]], axis=1)
    largest = np.argmax(np.abs(wxyz), axis=1)
    wxyz = wxyz * np.where(wxyz[np.arange(n), largest] < 0, -1.0, 1.0)[:, None]
    rot = largest.astype(np.uint64) << 30
    for slot in range(3):
        idx = np.array([[j for j in range(4) if j != L][slot] for L in largest])
        v = wxyz[np.arange(n), idx] / math.sqrt(2) + 0.5
        rot |= np.clip(np.round(v * 1023), 0, 1023).astype(np.uint64) << np.uint64(20 - 10 * slot)
    chunk_cols = []
    names = ["min_x", "min_y", "min_z", "max_x", "max_y", "max_z", "min_scale_x", "min_scale_y", "min_scale_z",
             "max_scale_x", "max_scale_y", "max_scale_z"]
    vals = [cmin[:, 0], cmin[:, 1], cmin[:, 2], cmax[:, 0], cmax[:, 1], cmax[:, 2],
            smin[:, 0], smin[:, 1], smin[:, 2], smax[:, 0], smax[:, 1], smax[:, 2]]
    if color_ranges:
        names += ["min_r", "min_g", "min_b", "max_r", "max_g", "max_b"]
        vals += [rmin[:, 0], rmin[:, 1], rmin[:, 2], rmax[:, 0], rmax[:, 1], rmax[:, 2]]
    chunk_cols = [(nm, "f4", v) for nm, v in zip(names, vals)]
    vert_cols = [("packed_position", "u4", pos), ("packed_rotation", "u4", rot), ("packed_scale", "u4", scl),
                 ("packed_color", "u4", col)]
    elements = [("chunk", chunks, [(nm, "float") for nm, _, _ in chunk_cols]),
                ("vertex", n, [(nm, "uint") for nm, _, _ in vert_cols])]
    body = _records(chunk_cols, little) + _records(vert_cols, little)
    deg = d["sh_degree"]
    if sh and deg:
        k = (deg + 1) ** 2 - 1
        rest = np.clip(np.trunc((d["colors"][:, 1:].astype(np.float64) / 8 + 0.5) * 256), 0, 255)  # encodeCompressedSh
        sh_cols = [(f"f_rest_{ch * k + j}", "u1", rest[:, j, ch]) for ch in range(3) for j in range(k)]
        elements.append(("sh", n, [(nm, "uchar") for nm, _, _ in sh_cols]))
        body += _records(sh_cols, little)
    return _header(elements, little) + body
