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


@pytest.mark.parametrize("pad", [0, 1, 2, 3])
def test_records_at_every_alignment(ctx, pad):
    # a count that leaves the last warp of 32 records and the last block part-filled;
    # the comment's length moves the records' start through the four byte offsets
    d = syn.mixture_table(1003, seed=7, sh_degree=3)
    raw = pf.standard_ply(d, comment="x" * pad)
    _check(raw)
    _check(raw, device_bytes=True)


def test_records_too_long_to_stage(ctx):
    # 59 floats and 130 doubles: 1276-byte records, decoded in place a thread per record
    d = syn.mixture_table(700, seed=13, sh_degree=3)
    raw = pf.standard_ply(d, extra_doubles=130)
    _check(raw)
    _check(raw, sh_degree=2, device_bytes=True)


def test_header_longer_than_the_first_read(ctx):
    # a device file whose header (a 6000-character comment) ends past the first 4 KB read
    raw = pf.standard_ply(syn.mixture_table(300, seed=4, sh_degree=1), comment="c" * 6000)
    assert raw.index(b"end_header") > 4096
    _check(raw, device_bytes=True)
    assert rb.ply_info(torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda())["count"] == 300


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_device_bytes_off_a_word_boundary(ctx, offset):
    raw = pf.standard_ply(syn.mixture_table(777, seed=8, sh_degree=2))
    buf = torch.zeros(len(raw) + 8, dtype=torch.uint8, device="cuda")
    buf[offset:offset + len(raw)] = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda()
    table, cols = rb.decode_ply(buf[offset:offset + len(raw)])
    ref = orc.ply_decode(raw)
    np.testing.assert_array_equal(host(cols["colors"]).reshape(ref["colors"].shape), ref["colors"].astype(np.float32))
    np.testing.assert_array_equal(host(cols["centers"]).reshape(-1, 3), ref["centers"].astype(np.float32))


@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
def test_every_row_width(ctx, degree):
    # rows of 3, 12, 27, 48 and 75 floats from an SH-4 file, in both byte orders
    d = syn.mixture_table(2500, seed=9, sh_degree=4)
    _check(pf.standard_ply(d), sh_degree=degree)
    _check(pf.standard_ply(d, little=False), sh_degree=degree)


@pytest.mark.parametrize("degree", [1, 3])
def test_colour_rows_off_a_16_byte_boundary(ctx, degree):
    # rows of 12 and 48 floats into a colour column that is 4- but not 16-byte aligned
    import ctypes
    raw = pf.standard_ply(syn.mixture_table(1500, seed=12, sh_degree=3))
    ref = orc.ply_decode(raw, degree)
    n, row = 1500, ((degree + 1) ** 2) * 3
    cols = torch.zeros(n * row + 4, device="cuda")
    data = np.frombuffer(raw, dtype=np.uint8)
    rb.default_context(0).call("rdx_decode_ply", ctypes.c_void_p(data.ctypes.data), len(raw), degree, None, None,
                               None, None, ctypes.c_void_p(cols.data_ptr() + 4))
    torch.cuda.synchronize()
    got = host(cols[1:1 + n * row]).reshape(ref["colors"].shape)
    np.testing.assert_array_equal(got, ref["colors"].astype(np.float32))
    assert float(cols[0]) == 0.0 and np.all(host(cols[1 + n * row:]) == 0.0)


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
