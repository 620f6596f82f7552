"""Decoders of the ray methods' words and the word-by-word comparison of two
projections, for the ray-method tests.

The decoders restate the reference's draw-side readers: decodeCenter,
decodeBound and decodeLogScale (src/render/projection.tsl.ts:305-307, 335-347,
362-368) and the words' positions (src/render/projections.tsl.ts:5-17, 310-314, 435-439).
"""
import math

import numpy as np

from oracle import oracle as orc

# head words, words per eye
LAYOUT = orc.RAY_WORDS


def eye_words(words, method, eye):
    h, w = LAYOUT[method]
    return words[:, h + eye * w: h + (eye + 1) * w]


def drawn(words, method, eye):
    """An eye draws a splat when its second word is nonzero (projections.tsl.ts:17)."""
    return eye_words(words, method, eye)[:, 1] != 0


def decode_center(words, method):
    """decodeCenter (projection.tsl.ts:335-347): the head-space centre of each row."""
    last = words[:, 5] if method != "raygs" else words[:, 3]
    dirw, dist = words[:, 0].astype(np.int64), words[:, 1].view(np.float32).astype(np.float64)
    last = last.astype(np.int64)
    qx = ((dirw & 0xFFFF) << 4) | ((last >> 24) & 15)
    qy = ((dirw >> 16) << 4) | (last >> 28)
    x = qx / 0xFFFFF * 2.0 - 1.0
    y = qy / 0xFFFFF * 2.0 - 1.0
    z = 1.0 - np.abs(x) - np.abs(y)
    t = np.maximum(-z, 0.0)
    x = x + np.where(x >= 0, -t, t)
    y = y + np.where(y >= 0, -t, t)
    v = np.stack([x, y, z], 1)
    return v / np.linalg.norm(v, axis=1, keepdims=True) * dist[:, None]


def decode_bound(w0, w1):
    """decodeBound (projection.tsl.ts:362-368): ndc [n][2], angle [n], scales [n][2]."""
    w0 = w0.astype(np.int64)
    w1 = w1.astype(np.int64)
    fixed16 = lambda c: c / 65535.0 * 4.0 - 2.0
    log_scale = lambda c: 2.0 ** ((c - 1) / 2046.0 * 16.0 - 4.0)
    ndc = np.stack([fixed16(w0 & 0xFFFF), fixed16(w0 >> 16)], 1)
    angle = (w1 & 1023) / 1024.0 * math.pi
    scales = np.stack([log_scale((w1 >> 10) & 0x7FF), log_scale(w1 >> 21)], 1)
    return ndc, angle, scales


def compare(gpu_words, ref_words, gpu_keys, ref_keys, method, eyes):
    """Drawn-eye disagreements, key mismatches, and the share of words that
    differ among rows both sides draw the same way (per eye)."""
    g = np.asarray(gpu_words).view(np.uint32)
    r = np.asarray(ref_words)
    disagree = 0
    same = np.ones(len(r), dtype=bool)
    for e in range(eyes):
        dg, dr = drawn(g, method, e), drawn(r, method, e)
        disagree += int((dg != dr).sum())
        same &= dg == dr
    diff = g[same] != r[same]
    out = {
        "rows": len(r),
        "drawn": int(sum(drawn(r, method, e).sum() for e in range(eyes))),
        "drawn_disagreements": disagree,
        "key_mismatches": int((np.asarray(gpu_keys).view(np.uint32) != np.asarray(ref_keys)).sum()),
        "word_mismatch_share": float(diff.mean()) if diff.size else 0.0,
        "word_mismatches_by_position": diff.sum(0).tolist(),
    }
    if method == "raygs":
        # c^2 as float32 bits: within one float32 step of the float64 value's rounding
        for e in range(eyes):
            col = LAYOUT[method][0] + e * LAYOUT[method][1] + 1
            m = same & (r[:, col] != 0)
            a = g[m, col].view(np.float32).astype(np.float64)
            b = r[m, col].view(np.float32).astype(np.float64)
            out[f"c2_rel_{e}"] = float(np.max(np.abs(a - b) / np.abs(b))) if m.any() else 0.0
    return out
