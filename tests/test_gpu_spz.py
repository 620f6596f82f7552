"""SPZ files decoded on the GPU against the oracle's reader: every column
bit-exact to the float32 rounding of the oracle's float64 values, for gzip
versions 1 to 4, several gzip members with trailers, SPZ 4 (NGSP) with
extension records, SH degrees 0 to 4 and a lower output degree; the header
view, the reference's error texts, and a decoded file drawn by a frame with
the oracle's order."""
import struct

import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests import spz_fixtures as sf
from tests.parity import host, u32

pytestmark = pytest.mark.gpu


def _check(raw, sh_degree=-1):
    table, cols = rb.decode_spz(raw, sh_degree)
    ref = orc.spz_decode(raw, sh_degree)
    for k in ("centers", "log_scales", "quats", "opacities", "colors"):
        np.testing.assert_array_equal(host(cols[k]).reshape(ref[k].shape), ref[k].astype(np.float32), err_msg=k)
    return table, ref


@pytest.mark.parametrize("version", [1, 2, 3, 4])
def test_gzip_versions(ctx, version):
    d = syn.mixture_table(20_000, seed=version, sh_degree=3)
    raw = sf.gzip_spz(d, version=version)
    _check(raw)
    info = rb.spz_info(raw)
    assert info == {"count": 20_000, "version": version, "sh_degree": 3, "fractional_bits": 12, "flags": 1,
                    "container": "gzip"}


@pytest.mark.parametrize("degree", [0, 1, 2, 4])
def test_sh_degrees_lower_output_and_members(ctx, degree):
    d = syn.mixture_table(7_000, seed=40 + degree, sh_degree=degree)
    raw = sf.gzip_spz(d, fractional_bits=16, members=2, trailer=bytes(7_000 * 6), flags=0x81)
    _check(raw)
    if degree > 0:
        _check(raw, sh_degree=degree - 1)


def test_more_splats_than_one_sweep_of_the_grid(ctx):
    # 1.25M splats: the decode's warps (4736 blocks of 8) take a second tile each
    d = syn.mixture_table(1_250_000, seed=60, sh_degree=1)
    _check(sf.gzip_spz(d, level=1))


def test_ngsp_container(ctx):
    if orc.zstd_lib() is None:
        pytest.skip("libzstd is not on this machine")
    d = syn.mixture_table(15_000, seed=50, sh_degree=3)
    records = sf.record(0xADBE0003, struct.pack("<I", 6)) + sf.record(0x12340001, bytes(3))
    raw = sf.ngsp_spz(d, records=records)
    _check(raw)
    assert rb.spz_info(raw)["container"] == "ngsp"
    _check(sf.ngsp_spz(syn.mixture_table(333, seed=51, sh_degree=0)))


def test_errors_carry_the_reference_texts(ctx):
    d = syn.mixture_table(100, seed=60, sh_degree=1)
    raw = sf.gzip_spz(d)
    with pytest.raises(rb.RadixError, match="Invalid SPZ file"):
        rb.decode_spz(b"not an spz file at all")
    with pytest.raises(rb.RadixError, match="ended unexpectedly"):
        rb.decode_spz(raw[:len(raw) // 2])
    import gzip
    body = gzip.decompress(raw)
    with pytest.raises(rb.RadixError, match="Unsupported SPZ version 9 or SH degree 1"):
        rb.spz_info(gzip.compress(body[:4] + struct.pack("<I", 9) + body[8:]))
    with pytest.raises(rb.RadixError, match="SH degree 1, not 2"):
        rb.decode_spz(raw, sh_degree=2)
    with pytest.raises(rb.RadixError, match="host memory"):
        rb.decode_spz(torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda())
    if orc.zstd_lib() is not None:
        ng = sf.ngsp_spz(d)
        with pytest.raises(rb.RadixError, match="bytes after its last stream"):
            rb.decode_spz(ng + b"\0\0")
        with pytest.raises(rb.RadixError, match="streams, 6 expected"):
            rb.spz_info(ng[:15] + bytes([4]) + ng[16:])
    # the context still works after the errors
    _check(raw)


def test_decoded_file_drawn_by_a_frame(ctx):
    d = syn.mixture_table(150_000, seed=61, sh_degree=3)
    table, ref = _check(sf.gzip_spz(d))
    cam = syn.scale_camera()
    res = rb.frame([rb.SplatObject(table)], cam, None, 32)
    host_table = {k: ref[k].astype(np.float32) for k in ("centers", "log_scales", "quats", "opacities", "colors")}
    host_table["sh_degree"] = 3
    o = orc.project([rb.SplatObject(rb.Table.from_dict(host_table))], cam, None, 32, cull_keys=True)
    n = d["centers"].shape[0]
    expected, visible = orc.sort(o["keys"], n, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"])[:n], expected[:n])
