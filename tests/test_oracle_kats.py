"""The oracle against the reference's own known answers (tests/golden/kats.json,
each entry citing the reference check it restates). CPU only."""
import json
import math
import os

import numpy as np
import pytest

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import camera as cm
from radix_b200.synthetic import Mulberry32

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kats.json")))
BITS = (16, 24, 32)


def test_sort_keys_monotonic_invalid_and_known_answer():
    k = KATS["sort_keys_monotonic"]
    for bits in BITS:
        keys = [orc.sort_key(d, bits) for d in k["distances"]]
        assert all(keys[i] <= keys[i - 1] for i in range(1, len(keys))), bits
        assert all(key < orc.lib().orc_valid_max(bits) + 1 for key in keys)
        for d in (math.inf, math.nan, -math.inf):
            assert orc.sort_key(d, bits) == rb.SortKeys.invalid(bits)
    assert orc.sort_key(1.0, 32) == k["key_of_1_at_32"] == 0xC07FFFFF


def test_invalid_and_valid_max_constants():
    for bits in BITS:
        assert orc.lib().orc_invalid_key(bits) == rb.SortKeys.invalid(bits)
        assert orc.lib().orc_valid_max(bits) == rb.SortKeys.valid_max(bits)


def _stability_case(seed=12345):
    k = KATS["sort_stability"]
    rng = Mulberry32(seed)
    u = rng.uniform(k["count"])
    d = np.round(u * 1000) / 10
    d[:: k["infinite_every"]] = np.inf
    return d


def test_sort_stable_invalid_last_same_order_every_width():
    d = _stability_case()
    n = d.size
    finite = np.flatnonzero(np.isfinite(d))
    expected = finite[np.lexsort((finite, -d[finite]))]  # far to near, ties by index
    for bits in BITS:
        keys = orc.sort_keys(d, bits)
        ordering, visible = orc.sort(keys, n, bits)
        assert visible == expected.size
        np.testing.assert_array_equal(ordering[:visible], expected)
        assert not np.isfinite(d[ordering[visible:n]]).any()


def test_sort_short_ordering_raises():
    with pytest.raises(ValueError, match="ordering holds 3 of 5 indices"):
        orc.sort(np.arange(5, dtype=np.uint32), 5, 32, ordering_len=3)


def test_sort_16bit_uses_low_bits_and_visible_layouts():
    # sort1x16 keys & 0xffff; visible excludes the top digit of each layout
    keys = np.array([0x1FFFF, 0x0001, 0xFFFF, 0x10000], dtype=np.uint32)
    o, v = orc.sort(keys, 4, 16)
    assert list(o[:4]) == [3, 1, 0, 2] and v == 2
    keys32 = np.array([0xFFFF0000, 0xFF000000, 0xFFFFFFFF, 5], dtype=np.uint32)
    o, v = orc.sort(keys32, 4, 32)
    assert list(o[:4]) == [3, 1, 0, 2] and v == 2  # top 16 bits all ones: 2 hidden
    keys24 = np.array([0xFFF800, 0xFFF7FF, 3], dtype=np.uint32)
    o, v = orc.sort(keys24, 3, 24)
    assert list(o[:3]) == [2, 1, 0] and v == 2  # top 13 bits all ones: 1 hidden


def test_sh_band1_known_answers():
    k = KATS["sh_band1"]
    c = np.zeros(72)
    for i, val in k["coeff_index_value"]:
        c[i] = val
    axes = {"x": (1, 0, 0), "y": (0, 1, 0), "z": (0, 0, 1)}
    for axis, channel, factor in k["expect"]:
        out = orc.sh_evaluate(c, axes[axis], 1)
        assert abs(out[channel] - factor * k["k"]) < k["tolerance"]


def _real_sh(l, m, d):
    """Real SH from associated Legendre polynomials, Condon-Shortley phase."""
    am = abs(m)
    x = d[2]
    pmm = 1.0
    for i in range(1, am + 1):
        pmm *= -(2 * i - 1) * math.sqrt(max(0.0, 1 - x * x))
    p = pmm
    if l > am:
        low = pmm
        p = x * (2 * am + 1) * pmm
        for n in range(am + 2, l + 1):
            low, p = p, ((2 * n - 1) * x * p - (n + am - 1) * low) / (n - am)
    ratio = 1.0
    for i in range(l - am + 1, l + am + 1):
        ratio /= i
    k = math.sqrt((2 * l + 1) / (4 * math.pi) * ratio)
    phi = math.atan2(d[1], d[0])
    if m == 0:
        return k * p
    return math.sqrt(2) * k * (math.cos(m * phi) if m > 0 else math.sin(am * phi)) * p


def test_sh_bands_match_real_sh():
    k = KATS["sh_legendre"]
    rng = Mulberry32(7)
    worst = 0.0
    done = 0
    while done < k["directions"]:
        v = rng.uniform(3) * 2 - 1
        nv = np.linalg.norm(v)
        if not (0.1 < nv <= 1):
            continue
        d = v / nv
        done += 1
        for l in range(1, 5):
            for m in range(-l, l + 1):
                idx = l * l - 1 + m + l
                c = np.zeros(72)
                c[idx * 3 + 1] = 1
                worst = max(worst, abs(orc.sh_evaluate(c, d, 4)[1] - _real_sh(l, m, d)))
                assert orc.sh_evaluate(c, d, l - 1)[1] == 0
    assert worst < k["tolerance"]


def _random_unit(rng):
    while True:
        v = rng.uniform(3) * 2 - 1
        n = np.linalg.norm(v)
        if 0.1 < n <= 1:
            return v / n


def _quat_angle(a, b):
    d = abs(float(np.dot(a / np.linalg.norm(a), b / np.linalg.norm(b))))
    return math.degrees(2 * math.acos(min(1.0, d)))


def test_ext_codec_budgets():
    k = KATS["ext_budgets"]
    rng = Mulberry32(11)
    worst_rot = 0.0
    for _ in range(2000):
        rgb = (rng.uniform(3) - 0.5) * 4
        back = orc.decode_ext_rgb(orc.encode_ext_rgb(rgb))
        assert np.max(np.abs(back - rgb)) <= np.max(np.abs(rgb)) * k["rgb_of_max"] + 1e-9
        axis = _random_unit(rng)
        angle = float(rng.uniform(1)[0]) * 2 * math.pi
        q = np.array([*(axis * math.sin(angle / 2)), math.cos(angle / 2)])
        worst_rot = max(worst_rot, _quat_angle(orc.decode_quat_oct32(orc.encode_quat_oct32(q)), q))
    assert worst_rot <= k["rotation_degrees"]
    worst_small = 0.0
    for _ in range(2000):
        axis = _random_unit(rng)
        half = float(rng.uniform(1)[0]) * 2 * math.pi / 180 / 2
        q = np.array([*(axis * math.sin(half)), math.cos(half)])
        worst_small = max(worst_small, _quat_angle(orc.decode_quat_oct32(orc.encode_quat_oct32(q)), q))
    assert worst_small <= k["small_turn_degrees"]


def test_identity_and_zero_quaternions():
    for q in ([0, 0, 0, 1], [0, 0, 0, 0]):
        assert list(orc.decode_quat_oct32(orc.encode_quat_oct32(q))) == [0, 0, 0, 1]


def test_half_codec():
    for h in (0x0000, 0x0001, 0x03FF, 0x0400, 0x3C00, 0x7BFF, 0x8001, 0xBC00, 0xC000):
        assert orc.encode_half(orc.decode_half(h)) == h
    assert orc.decode_half(0x7C00) == math.inf and math.isnan(orc.decode_half(0x7E00))
    assert orc.encode_half(1.0 + 2 ** -11) == 0x3C00  # ties to even
    assert orc.encode_half(1.0 + 3 * 2 ** -11) == 0x3C02


def _decode_depth20(code):
    """decodeDepth20 (src/render/projection.tsl.ts:290): the float bits above 2^-14, negated."""
    bits = np.uint32((int(code) << 8) + (113 << 23))
    return -float(bits.view(np.float32))


def test_depth20_angle12_codec_budgets():
    k = KATS["codecs_depth_angle"]
    n = 1000
    for i in range(n + 2):
        t = i / (n - 1)
        depth = 1e-6 if i == n else (1e7 if i == n + 1 else 2 ** (math.log2(1e-3) + t * (math.log2(1e5) - math.log2(1e-3))))
        back = -_decode_depth20(orc.lib().orc_encode_depth20(-depth))
        expected = min(max(depth, 2 ** -14), 2 ** 18)
        assert abs(back / expected - 1) <= k["depth_rel"] * 1.01
        if i < n:
            angle = t * math.pi
            code = orc.lib().orc_encode_angle12(angle)
            turn = abs(code / 4096 * math.pi - angle) % math.pi
            assert min(turn, math.pi - turn) <= k["angle"] * 1.01


def test_matrix_inverse_and_product_match_numpy():
    rng = Mulberry32(3)
    for _ in range(20):
        m = rng.normal(16)
        out = np.zeros(16)
        assert orc.lib().orc_mat4_invert(m.ctypes.data, out.ctypes.data) == 1
        np.testing.assert_allclose(out.reshape(4, 4).T, np.linalg.inv(m.reshape(4, 4).T), rtol=1e-9, atol=1e-9)
        b = rng.normal(16)
        prod = np.zeros(16)
        orc.lib().orc_mat4_mul(m.ctypes.data, b.ctypes.data, prod.ctypes.data)
        np.testing.assert_allclose(prod.reshape(4, 4).T, m.reshape(4, 4).T @ b.reshape(4, 4).T, rtol=1e-12)


def _test_camera(position, width=128, height=64):
    """makeCamera of test/gpu/renderUtils.ts:63-70: fov 60, near 0.1, far 100, looking down -z."""
    view = cm.invert(cm.translation(*position))
    proj = cm.perspective(60.0, width / height, 0.1, 100.0)
    return rb.Camera(view, [(view, proj, False)], width, height)


def _splat_table(centers, scales, quats=None, rgb=None, opacities=None):
    n = len(centers)
    quats = np.tile([0, 0, 0, 1.0], (n, 1)) if quats is None else np.asarray(quats)
    rgb = np.ones((n, 1, 3)) if rgb is None else np.asarray(rgb).reshape(n, 1, 3)
    opacities = np.ones(n) if opacities is None else np.asarray(opacities)
    return dict(centers=np.asarray(centers, dtype=np.float32), log_scales=np.log(np.asarray(scales)).astype(np.float32),
                quats=quats.astype(np.float32), opacities=opacities.astype(np.float32), colors=rgb.astype(np.float32),
                sh_degree=0)


def random_test_splats(count, seed):
    """Splats in a box in front of a camera at the origin (renderUtils.ts:43-54 distributions)."""
    rng = Mulberry32(seed)
    u = rng.uniform(count * 13).reshape(count, 13)
    centers = np.stack([(u[:, 0] - 0.5) * 4, (u[:, 1] - 0.5) * 3, -2 - u[:, 2] * 6], axis=1)
    scales = np.stack([0.01 + u[:, 3] * 0.1, 0.01 + u[:, 4] * 0.1, 0.01 + u[:, 5] * 0.05], axis=1)
    rgb = u[:, 6:9]
    opac = 0.2 + u[:, 9] * 0.8
    axis = u[:, 10:13] - 0.5
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    angle = rng.uniform(count) * 2 * math.pi
    quats = np.concatenate([axis * np.sin(angle / 2)[:, None], np.cos(angle / 2)[:, None]], axis=1)
    return _splat_table(centers, scales, quats, rgb, opac)


def test_ewa_bound_matches_the_reference_cpu_ewa():
    k = KATS["ewa_bound"]
    data = random_test_splats(k["splats"], 3)
    cam = _test_camera(k["camera"]["position"])
    params = rb.SplatParams(blur_amount=0.0)
    out = orc.project([rb.SplatObject(rb.Table.from_dict(data))], cam, params, 32)
    P = cam.eyes[0][1]
    fx, fy = 64 * P[0], 32 * P[5]
    view = cam.eyes[0][0].reshape(4, 4).T
    std = math.sqrt(8)
    checked = 0
    for i in range(k["splats"]):
        if not out["visible"][0, i]:
            continue
        c = view @ np.append(data["centers"][i].astype(np.float64), 1.0)
        x, y, z, w = data["quats"][i].astype(np.float64)
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        M = view[:3, :3] @ R @ np.diag(np.exp(data["log_scales"][i].astype(np.float64)))
        cov = M @ M.T
        J = np.array([[fx / c[2], 0, -fx * c[0] / c[2] ** 2], [0, fy / c[2], -fy * c[1] / c[2] ** 2], [0, 0, 0]])
        cov2 = J @ cov @ J.T
        a, b, d = cov2[0, 0], cov2[0, 1], cov2[1, 1]
        avg = (a + d) / 2
        delta = math.sqrt(max(0.0, avg * avg - (a * d - b * b)))
        major, minor = std * math.sqrt(avg + delta), std * math.sqrt(max(avg - delta, 0))
        s1, s2 = out["radii"][0, i, :2]
        # the params are float32 (maxStdDev = fround(sqrt 8)): far inside the 1% / 2% of the check
        assert abs(s1 / major - 1) < 1e-6 and abs(s2 / minor - 1) < 1e-5
        checked += 1
    assert checked > 100


def test_culling_and_cull_keys():
    k = KATS["culling"]
    data = _splat_table(k["centers"], [[k["scale"]] * 3] * 4, opacities=k["opacities"])
    cam = _test_camera((0, 0, 0))
    obj = [rb.SplatObject(rb.Table.from_dict(data))]
    for cull_keys, expected in ((True, k["invalid_cull_keys"]), (False, k["invalid_no_cull_keys"])):
        out = orc.project(obj, cam, rb.SplatParams(), 32, cull_keys)
        assert [not bool(v) for v in out["visible"][0]] == k["culled"]
        assert [int(key) == rb.SortKeys.invalid(32) for key in out["keys"]] == expected


def test_sort_guard():
    k = KATS["sort_guard"]
    data = _splat_table(k["centers"], [[k["scale"]] * 3] * 4)
    cam = _test_camera((0, 0, 0))
    obj = [rb.SplatObject(rb.Table.from_dict(data))]
    for guard, expected in ((0.0, k["valid_guard0"]), (k["guard"], k["valid_guard"])):
        out = orc.project(obj, cam, rb.SplatParams(sort_guard=guard), 24, False)
        assert [int(key) != rb.SortKeys.invalid(24) for key in out["keys"]] == expected


def test_keys_are_sort_keys_of_the_head_distance():
    data = random_test_splats(500, 3)
    cam = _test_camera((-0.03, 0, 0))
    out = orc.project([rb.SplatObject(rb.Table.from_dict(data))], cam, rb.SplatParams(), 32, False)
    d = np.linalg.norm(data["centers"].astype(np.float64) - np.array([-0.03, 0, 0]), axis=1)
    for bits in BITS:
        keys = orc.project([rb.SplatObject(rb.Table.from_dict(data))], cam, rb.SplatParams(), bits, False)["keys"]
        ref = orc.sort_keys(d, bits)
        # float64 head distance on both sides: at most one float32 ulp of distance apart
        assert np.max(np.abs(keys.astype(np.int64) - ref.astype(np.int64))) <= 1
    assert out["keys"].dtype == np.uint32


def test_ext_table_decodes_close_to_raw():
    data = random_test_splats(300, 5)
    a, b, sh = orc.encode_ext(data)
    ext = rb.Table.ext(a, b, sh, 0)
    cam = _test_camera((0, 0, 0))
    raw_out = orc.project([rb.SplatObject(rb.Table.from_dict(data))], cam, rb.SplatParams(), 32, False)
    ext_out = orc.project([rb.SplatObject(ext)], cam, rb.SplatParams(), 32, False)
    vis = raw_out["visible"][0].astype(bool) & ext_out["visible"][0].astype(bool)
    assert vis.sum() > 200
    # half-float log scales and an 8-bit colour: within the codec budgets
    np.testing.assert_allclose(ext_out["mean2d"][0][vis], raw_out["mean2d"][0][vis], rtol=1e-6)
    np.testing.assert_allclose(ext_out["rgb"][0][vis], raw_out["rgb"][0][vis], atol=1.0 / 255 + 1e-9)
