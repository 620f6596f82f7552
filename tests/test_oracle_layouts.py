"""The oracle's packed and cov splat codecs and its SH codecs / palettes,
against the budgets the reference's own checks hold them to:
packed splats within their encoding ranges (scripts/check-core.ts:440-469),
cov splats' encoding bounds (check-core.ts:402-425), the SH codecs' round
trips within 0.2 / 0.4 8-bit steps RMS and the packed prefix property
(check-core.ts:1265-1291). Fixtures are seeded, with the distributions of
those checks (randomSplat, shValues)."""
import math

import numpy as np
import pytest

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200.synthetic import Mulberry32

N = 2000


def _random_splats(n, seed=7, sh_degree=0, coeffs=None):
    """randomSplat's distributions (check-core.ts:67-79) as a raw table dict."""
    r = Mulberry32(seed)
    centers = (r.uniform(3 * n).reshape(n, 3) - 0.5) * 200.0
    log_scales = r.uniform(3 * n).reshape(n, 3) * 9.0 - 6.0
    q = r.normal(4 * n).reshape(n, 4)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    rgb = r.uniform(3 * n).reshape(n, 3) * 4.0 - 1.0
    opac = r.uniform(n) * (255.0 / 128.0)
    k = (sh_degree + 1) ** 2 - 1
    colors = np.zeros((n, 1 + k, 3))
    colors[:, 0] = rgb
    if k:
        colors[:, 1:] = coeffs.reshape(n, k, 3)
    return dict(centers=centers.astype(np.float32), log_scales=log_scales.astype(np.float32),
                quats=q.astype(np.float32), opacities=opac.astype(np.float32), colors=colors.astype(np.float32),
                sh_degree=sh_degree)


def _quat_angle(a, b):
    d = min(1.0, abs(float(np.dot(a, b)) / (np.linalg.norm(a) * np.linalg.norm(b))))
    return 2.0 * math.degrees(math.acos(d))


def test_packed_splats_within_their_encoding_ranges():
    d = _random_splats(N)
    r = Mulberry32(11)
    d["colors"][:, 0] = r.uniform(3 * N).reshape(N, 3).astype(np.float32)  # inside [rgbMin, rgbMax]
    d["opacities"] = r.uniform(N).astype(np.float32)
    d["centers"] = ((r.uniform(3 * N).reshape(N, 3) - 0.5) * 20.0).astype(np.float32)
    enc = rb.Table.PACKED_ENCODING
    t = rb.Table.packed(orc.encode_packed(d, enc))
    rgb_min, rgb_max, ln_min, ln_max = enc
    worst = 0.0
    for i in range(N):
        s = orc.load_splat(t, i)
        assert abs(s["rgb"][1] - d["colors"][i, 0, 1]) <= (rgb_max - rgb_min) / 510 + 1e-6, i
        assert abs(s["opacity"] - d["opacities"][i]) <= 1 / 510 + 1e-6, i
        c = float(d["centers"][i, 1])
        assert abs(s["center"][1] - c) <= abs(c) * 2 ** -11 + 2 ** -25, i
        sx = math.exp(float(d["log_scales"][i, 0]))
        if math.exp(ln_min) <= sx <= math.exp(ln_max):
            assert abs(math.log(s["scales"][0]) - math.log(sx)) <= (ln_max - ln_min) / 254 / 2 + 1e-6, i
        worst = max(worst, _quat_angle(s["quat"], d["quats"][i].astype(np.float64)))
    assert worst <= 2.0, worst  # angle step pi / 255 plus the 8-bit axis


def _ln_half_bound(v):
    # |ln v| rounded to a half float: half an ulp of the half, relative 2^-11
    return abs(math.log(v)) * 2 ** -11 + 2 ** -25


def test_cov_splats_within_their_encoding_bounds():
    d = _random_splats(N, seed=9)
    a, b = orc.encode_cov(d)
    t = rb.Table.cov(a, b)
    raw = rb.Table.from_dict(d)
    for i in range(N):
        s = orc.load_splat(t, i)
        r = orc.load_splat(raw, i)
        q = r["quat"] / np.linalg.norm(r["quat"])
        x, y, z, w = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        M = R * r["scales"]
        C = M @ M.T
        c = {"xx": C[0, 0], "yy": C[1, 1], "zz": C[2, 2], "xy": C[0, 1], "xz": C[0, 2], "yz": C[1, 2]}
        got = dict(zip(("xx", "yy", "zz", "xy", "xz", "yz"), s["cov"]))
        for key, p, q_ in (("xy", "xx", "yy"), ("xz", "xx", "zz"), ("yz", "yy", "zz")):
            pa, pb = c[p], c[q_]
            corr = abs(c[key]) / math.sqrt(pa * pb)
            bound = math.sqrt(pa * pb) * (2e-4 + corr * (_ln_half_bound(pa) + _ln_half_bound(pb)) / 2)
            assert abs(got[key] - c[key]) <= bound * 1.01, (i, key)
        assert abs(math.log(got["xx"]) - math.log(c["xx"])) <= _ln_half_bound(c["xx"]) * 1.01, i


def _sh_values(n, degree, seed=5):
    """shValues (check-core.ts:1235-1237)."""
    r = Mulberry32(seed)
    k = ((degree + 1) ** 2 - 1) * 3
    u = r.uniform(n * k).reshape(n, k)
    v = r.uniform(n * k).reshape(n, k)
    scale = np.where((np.arange(n) % 211 == 0)[:, None], 10.0, 0.4 * v)
    return ((u - 0.5) * scale).astype(np.float32)


@pytest.mark.parametrize("codec,budget", [("ext", 0.2), ("packed", 0.4)])
def test_sh_codecs_within_their_budgets(codec, budget):
    n = 4000
    for degree in (4, 3, 2, 1):
        vals = _sh_values(n, degree)
        d = _random_splats(n, seed=3, sh_degree=degree, coeffs=vals)
        words = orc.encode_sh(d, codec)
        a, b = orc.encode_cov(d)
        t = rb.Table.ext(a, b, orc.sh_channels(words), sh_degree=degree, sh_codec=codec)
        err = np.array([orc.load_splat(t, i)["sh"] for i in range(n)]) - vals.astype(np.float64)
        rms = math.sqrt((err ** 2).sum() / n / 3 / (4 * math.pi)) * 255
        assert rms <= budget, (codec, degree, rms)


def test_packed_sh_prefix_reads_as_a_lower_degree():
    vals4 = _sh_values(64, 4, seed=8)
    d4 = _random_splats(64, seed=2, sh_degree=4, coeffs=vals4)
    w4 = orc.encode_sh(d4, "packed")
    a, b = orc.encode_cov(d4)
    for degree in (1, 2, 3):
        k = ((degree + 1) ** 2 - 1) * 3
        d = _random_splats(64, seed=2, sh_degree=degree, coeffs=vals4[:, :k].copy())
        w = orc.encode_sh(d, "packed")
        hi = rb.Table.ext(a, b, orc.sh_channels(w4), sh_degree=degree, sh_codec="packed")
        lo = rb.Table.ext(a, b, orc.sh_channels(w), sh_degree=degree, sh_codec="packed")
        for i in range(64):
            np.testing.assert_array_equal(orc.load_splat(hi, i)["sh"], orc.load_splat(lo, i)["sh"])


@pytest.mark.parametrize("codec", ["ext", "packed"])
def test_palette_entries_read_as_per_splat_channels(codec):
    n, size = 500, 37
    vals = _sh_values(size, 3, seed=12)
    entries = _random_splats(size, seed=4, sh_degree=3, coeffs=vals)
    words = orc.encode_sh(entries, codec)
    stride = 1 << (words.shape[1] // 4 - 1).bit_length()  # ShPalette.strideOf: texels rounded up to a power of two
    labels = (np.arange(n) * 7 % size).astype(np.uint16)
    d = _random_splats(n, seed=6)
    a, b = orc.encode_cov(d)
    pal = rb.Table.ext(a, b, sh_degree=3, sh_codec=codec, palette=(orc.sh_palette(words, stride), labels, stride))
    per = rb.Table.ext(a, b, orc.sh_channels(np.ascontiguousarray(words[labels])), sh_degree=3, sh_codec=codec)
    for i in range(0, n, 7):
        np.testing.assert_array_equal(orc.load_splat(pal, i)["sh"], orc.load_splat(per, i)["sh"])
