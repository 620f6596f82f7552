"""PLY files decoded on the GPU against the oracle's reader (float32 of its
float64 values; an ulp allowed where a square root, division or exp
rounds), for standard files with SH and odd-sized properties, point clouds
and compressed files in both byte orders, from host and device bytes; and a
decoded file drawn by a frame with the oracle's order."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests import ply_fixtures as pf
from tests.parity import host, u32

pytestmark = pytest.mark.gpu


def _check(raw, sh_degree=-1, device_bytes=False):
    data = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda() if device_bytes else raw
    table, cols = rb.decode_ply(data, sh_degree)
    ref = orc.ply_decode(raw, sh_degree)
    for k in ("centers", "log_scales", "colors"):
        np.testing.assert_array_equal(host(cols[k]).reshape(ref[k].shape), ref[k].astype(np.float32), err_msg=k)
    for k in ("quats", "opacities"):
        g = host(cols[k]).astype(np.float64).reshape(ref[k].shape)
        r = ref[k].astype(np.float32).astype(np.float64)
        assert np.all(np.abs(g - r) <= 2.0 ** -23 * np.maximum(np.abs(r), 2.0 ** -126)), k
    return table, ref


@pytest.mark.parametrize("little", [True, False])
def test_standard_files(ctx, little):
    d = syn.mixture_table(20_000, seed=3, sh_degree=3)
    _check(pf.standard_ply(d, little))
    _check(pf.standard_ply(d, little, extra_uchar=True), sh_degree=1)


def test_point_cloud_and_device_bytes(ctx):
    raw = pf.point_cloud_ply(5000, alpha=True)
    _check(raw)
    _check(raw, device_bytes=True)
    info = rb.ply_info(raw)
    assert info == {"count": 5000, "sh_degree": 0, "kind": "points"}


@pytest.mark.parametrize("little", [True, False])
def test_compressed_files(ctx, little):
    d = syn.mixture_table(10_000, seed=5, sh_degree=3)
    _check(pf.compressed_ply(d, little))
    _check(pf.compressed_ply(d, little, sh=False, color_ranges=False), device_bytes=True)


def test_errors_carry_the_reference_texts(ctx):
    d = syn.plain_table(100, seed=2)
    raw = pf.standard_ply(d)
    with pytest.raises(rb.RadixError, match="ended unexpectedly"):
        rb.decode_ply(raw[:-7])
    with pytest.raises(rb.RadixError, match="no vertex element"):
        rb.decode_ply(b"ply\nformat binary_little_endian 1.0\nelement face 0\nend_header\n")
    with pytest.raises(rb.RadixError, match="lacks"):
        rb.decode_ply(b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\nend_header\n" + bytes(4))


def test_decoded_file_drawn_by_a_frame(ctx):
    d = syn.mixture_table(200_000, seed=11, sh_degree=3)
    raw = pf.standard_ply(d)
    table, ref = _check(raw)
    cam = syn.scale_camera()
    res = rb.frame([rb.SplatObject(table)], cam, None, 32)
    host_table = {k: ref[k].astype(np.float32) for k in ("centers", "log_scales", "quats", "opacities", "colors")}
    host_table["sh_degree"] = 3
    o = orc.project([rb.SplatObject(rb.Table.from_dict(host_table))], cam, None, 32, cull_keys=True)
    n = d["centers"].shape[0]
    expected, visible = orc.sort(o["keys"], n, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"])[:n], expected[:n])
