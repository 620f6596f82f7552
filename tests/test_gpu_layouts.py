"""The projection of Radix's other splat layouts (packedSplats, covSplats,
extSplats) with SH in either codec (ext words, packed bytes), per splat or
from an ShPalette, against the float64 oracle reading the same words: keys
bit-exact, cull decisions equal, outputs within 1e-5; and a packed frame's
order bit-exact."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests.parity import TOLERANCE, compare_projection, host, to_cuda, u32

pytestmark = pytest.mark.gpu
ALL = ("mean2d", "conic", "depth", "opacity", "rgb", "radii", "words", "keys")


def _i32(a):
    return to_cuda(np.ascontiguousarray(a).view(np.int32))


def _tables(d, layout, codec, palette, encoding=rb.Table.PACKED_ENCODING):
    """(device table, host table) of the same words."""
    deg = d["sh_degree"]
    words = orc.encode_sh(d, codec) if deg else np.zeros((d["centers"].shape[0], 0), dtype=np.uint32)
    kw_h, kw_d = {}, {}
    if palette and deg:
        size = 97
        stride = 1 << (words.shape[1] // 4 - 1).bit_length()
        labels = (np.arange(words.shape[0]) * 13 % size).astype(np.uint16)
        entries = orc.sh_palette(np.ascontiguousarray(words[:size]), stride)
        kw_h["palette"] = (entries, labels, stride)
        kw_d["palette"] = (_i32(entries), to_cuda(labels.view(np.int16)), stride)
        sh_h, sh_d = (), ()
    else:
        sh_h = orc.sh_channels(words)
        sh_d = [_i32(c) for c in sh_h]
    if layout == "packed":
        p = orc.encode_packed(d, encoding)
        return (rb.Table.packed(_i32(p), encoding, sh_d, deg, codec, **kw_d),
                rb.Table.packed(p, encoding, sh_h, deg, codec, **kw_h))
    a, b = orc.encode_cov(d) if layout == "cov" else orc.encode_ext(d)[:2]
    make = rb.Table.cov if layout == "cov" else rb.Table.ext
    return make(_i32(a), _i32(b), sh_d, deg, codec, **kw_d), make(a, b, sh_h, deg, codec, **kw_h)


def _check(dev, hst, cam, params=None, bits=32):
    gpu = rb.project_collection([rb.SplatObject(dev)], cam, params, bits, cull_keys=True, outputs=ALL)
    ref = orc.project([rb.SplatObject(hst)], cam, params, bits, True)
    r = compare_projection(gpu, ref)
    print(r)
    assert r["drawn"] > 0
    assert r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, r
    for name, e in r["errors"].items():
        assert e < TOLERANCE, (name, e, r)
    return gpu, ref


@pytest.mark.parametrize("layout", ["packed", "cov", "ext"])
@pytest.mark.parametrize("codec", ["ext", "packed"])
@pytest.mark.parametrize("palette", [False, True])
def test_layouts_and_sh_codecs(ctx, layout, codec, palette):
    d = syn.mixture_table(40_000, seed=21, sh_degree=3)
    d["opacities"][::7] = np.float32(1.5)  # LoD opacities (ext and cov store up to 255/128)
    dev, hst = _tables(d, layout, codec, palette)
    _check(dev, hst, syn.scale_camera())


@pytest.mark.parametrize("degree", [0, 1, 2, 4])
def test_packed_layout_degrees_and_stereo(ctx, degree):
    d = syn.mixture_table(30_000, seed=22 + degree, sh_degree=degree)
    enc = (-0.5, 1.5, -10.0, 4.0)
    dev, hst = _tables(d, "packed", "packed", False, enc)
    _check(dev, hst, syn.scale_camera())
    _check(dev, hst, syn.stereo_camera())


def test_cov_layout_sort_guard_and_keys_pass(ctx):
    d = syn.mixture_table(30_000, seed=30, sh_degree=1)
    dev, hst = _tables(d, "cov", "ext", False)
    p = rb.SplatParams(sort_guard=0.2)
    cam = syn.scale_camera()
    gpu = rb.project_collection([rb.SplatObject(dev)], cam, p, 24, "keys")
    ref = orc.project([rb.SplatObject(hst)], cam, p, 24, False)
    np.testing.assert_array_equal(u32(gpu["keys"]), ref["keys"])


def test_packed_frame_order_bit_exact(ctx):
    d = syn.mixture_table(500_000, seed=31, sh_degree=3)
    dev, hst = _tables(d, "packed", "packed", True)
    cam = syn.scale_camera()
    res = rb.frame([rb.SplatObject(dev)], cam, None, 32)
    ref = orc.project([rb.SplatObject(hst)], cam, None, 32, cull_keys=True)
    n = d["centers"].shape[0]
    expected, visible = orc.sort(ref["keys"], n, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"])[:n], expected[:n])
