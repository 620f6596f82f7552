"""The oracle's PLY reader: the reference's own check of point clouds and SH
degree detection (scripts/check-core.ts:694-717), and round trips of
standard, point-cloud and compressed files written from synthetic tables in
both byte orders."""
import numpy as np
import pytest

from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests import ply_fixtures as pf


def test_reference_point_cloud_and_sh_degree():
    # check-core.ts:694-708: two points, the second at x = 2 with red 255
    header = ("ply\nformat binary_little_endian 1.0\nelement vertex 2\nproperty float x\nproperty float y\n"
              "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n").encode()
    body = bytearray(2 * 15)
    body[15:19] = np.float32(2).tobytes()
    body[15 + 12] = 255
    d = orc.ply_decode(header + bytes(body))
    assert d["kind"] == 1 and d["count"] == 2
    assert d["centers"][1, 0] == 2
    assert abs(d["colors"][1, 0, 0] - 1) <= 1 / 255 and d["colors"][1, 0, 1] == 0
    assert abs(np.exp(d["log_scales"][1, 0]) - 0.001) <= 1e-5
    # check-core.ts:710-717: 24 f_rest values are SH degree 2
    names = ["x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3", "opacity", "f_dc_0",
             "f_dc_1", "f_dc_2"] + [f"f_rest_{k}" for k in range(24)]
    sh = ("ply\nformat binary_little_endian 1.0\nelement vertex 1\n" + "\n".join(f"property float {n}" for n in names)
          + "\nend_header\n").encode() + bytes(len(names) * 4)
    assert orc.ply_decode(sh)["sh_degree"] == 2


@pytest.mark.parametrize("little", [True, False])
@pytest.mark.parametrize("degree", [0, 1, 3])
def test_standard_round_trip(little, degree):
    d = syn.mixture_table(3000, seed=degree + 1, sh_degree=degree)
    got = orc.ply_decode(pf.standard_ply(d, little, extra_uchar=degree == 1))
    assert got["kind"] == 0 and got["sh_degree"] == degree and got["count"] == 3000
    np.testing.assert_array_equal(got["centers"], d["centers"].astype(np.float64))
    np.testing.assert_array_equal(got["log_scales"], d["log_scales"].astype(np.float64))
    q = d["quats"].astype(np.float64)
    np.testing.assert_allclose(got["quats"], q / np.linalg.norm(q, axis=1, keepdims=True), atol=1e-7)
    np.testing.assert_allclose(got["opacities"], d["opacities"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(got["colors"][:, 0], d["colors"][:, 0], atol=1e-6)
    np.testing.assert_array_equal(got["colors"][:, 1:], d["colors"][:, 1:].astype(np.float64))


def test_point_cloud_alpha():
    raw = pf.point_cloud_ply(100, alpha=True)
    got = orc.ply_decode(raw)
    assert got["kind"] == 1 and got["sh_degree"] == 0
    assert (got["opacities"] >= 0).all() and (got["opacities"] <= 1).all()


@pytest.mark.parametrize("little", [True, False])
def test_compressed_round_trip(little):
    d = syn.mixture_table(1000, seed=9, sh_degree=2)
    got = orc.ply_decode(pf.compressed_ply(d, little))
    assert got["kind"] == 2 and got["sh_degree"] == 2
    # within the format's steps: 11/10-bit positions over a chunk's range, 8-bit colours and opacity
    span = np.ptp(d["centers"].reshape(-1, 3)[:256], axis=0)
    assert np.abs(got["centers"][:256] - d["centers"][:256]).max() <= span.max() / 1023 + 1e-6
    assert np.abs(got["opacities"] - d["opacities"]).max() <= 1 / 255 + 1e-6
    assert np.abs(got["colors"][:, 1:] - d["colors"][:, 1:]).max() <= 8 / 256 + 1e-6
    q = d["quats"].astype(np.float64)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    dots = np.abs((got["quats"] * q).sum(axis=1))
    assert np.degrees(2 * np.arccos(np.clip(dots, 0, 1))).max() < 1.0


def test_malformed_files_are_rejected():
    d = syn.plain_table(10, seed=1)
    raw = pf.standard_ply(d)
    with pytest.raises(ValueError):
        orc.ply_decode(raw[:-10])  # ends early
    with pytest.raises(ValueError):
        orc.ply_decode(b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n0\n")
