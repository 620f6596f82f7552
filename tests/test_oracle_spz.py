"""The SPZ oracle (oracle/oracle.c orc_spz_decode, oracle.py spz_unpack)
against the format's own rules, as the reference's SPZ checks hold them
(scripts/check-core.ts:825-1025: round trips of every version and container,
version 4 inside gzip read as version 3, extension records, SPZ 4 header
checks): files written here from synthetic tables decode back within each
field's quantisation step; malformed files fail with the reference's texts."""
import gzip
import math
import struct

import numpy as np
import pytest

from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests import spz_fixtures as sf

COLOR_STEP = sf.COLOR_SCALE / 255.0


def _unit(q):
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _within_steps(r, d, version, fb=12, degree=3):
    centre_step = 2.0 ** -fb if version > 1 else None
    if centre_step:
        assert np.abs(r["centers"] - d["centers"]).max() <= centre_step / 2 * (1 + 1e-9)
    else:  # halves: half an ulp of the half
        assert np.all(np.abs(r["centers"] - d["centers"]) <= np.maximum(np.abs(d["centers"]), 2.0 ** -14) * 2.0 ** -11)
    assert np.abs(r["log_scales"] - d["log_scales"]).max() <= 1 / 32 + 1e-9
    assert np.abs(r["opacities"] - d["opacities"]).max() <= 0.5 / 255 + 1e-9
    assert np.abs(r["colors"][:, 0] - d["colors"][:, 0]).max() <= COLOR_STEP / 2 + 1e-9
    k = sf.SH_VECTORS[degree]
    if k:
        assert np.abs(r["colors"][:, 1:1 + k] - d["colors"][:, 1:1 + k]).max() <= 1 / 256 + 1e-9
    dots = np.abs(np.sum(r["quats"] * _unit(d["quats"].astype(np.float64)), axis=1))
    # smallest three: 9-bit magnitudes; 3 bytes of x y z: about 1/255 per component
    assert dots.min() > (0.99999 if version >= 3 else 0.99)
    np.testing.assert_allclose(np.linalg.norm(r["quats"], axis=1), 1.0, atol=1e-12)


@pytest.mark.parametrize("version", [1, 2, 3, 4])
def test_gzip_versions_round_trip(version):
    d = syn.mixture_table(3000, seed=version, sh_degree=3)
    r = orc.spz_decode(sf.gzip_spz(d, version=version))
    assert (r["container"], r["version"], r["count"], r["sh_degree"]) == ("gzip", version, 3000, 3)
    _within_steps(r, d, version)


@pytest.mark.parametrize("degree", [0, 1, 2, 4])
def test_sh_degrees_and_fixed_point(degree):
    d = syn.mixture_table(1000, seed=10 + degree, sh_degree=degree)
    for fb in (8, 16):
        r = orc.spz_decode(sf.gzip_spz(d, fractional_bits=fb))
        _within_steps(r, d, 3, fb=fb, degree=degree)
    lower = orc.spz_decode(sf.gzip_spz(d), sh_degree=max(degree - 1, 0))
    full = orc.spz_decode(sf.gzip_spz(d))
    np.testing.assert_array_equal(lower["colors"], full["colors"][:, :lower["colors"].shape[1]])


def test_ngsp_container_and_records():
    z = orc.zstd_lib()
    if z is None:
        pytest.skip("libzstd is not on this machine")
    d = syn.mixture_table(2500, seed=21, sh_degree=3)
    records = sf.record(0xADBE0002, struct.pack("<3f", 0.25, 1.5, 3.0)) + sf.record(0x12340001, bytes(5))
    a = orc.spz_decode(sf.ngsp_spz(d, records=records))
    b = orc.spz_decode(sf.gzip_spz(d, version=3))
    assert a["container"] == "ngsp" and a["version"] == 4
    for k in ("centers", "log_scales", "quats", "opacities", "colors"):
        np.testing.assert_array_equal(a[k], b[k])
    # degree 0: five streams
    d0 = syn.mixture_table(100, seed=22, sh_degree=0)
    raw = sf.ngsp_spz(d0)
    assert raw[15] == 5 and orc.spz_decode(raw)["sh_degree"] == 0


def test_members_trailers_and_version_4_in_gzip():
    d = syn.mixture_table(1500, seed=30, sh_degree=2)
    one = orc.spz_decode(sf.gzip_spz(d, version=3))
    several = orc.spz_decode(sf.gzip_spz(d, version=3, members=3, trailer=bytes(1500 * 6), flags=0x81))
    v4 = orc.spz_decode(sf.gzip_spz(d, version=4))
    for k in ("centers", "log_scales", "quats", "opacities", "colors"):
        np.testing.assert_array_equal(one[k], several[k])
        np.testing.assert_array_equal(one[k], v4[k])


def test_smallest_three_known_answers():
    # largest = w (3): x, y, z from bits 20-29, 10-19, 0-9 (z lowest)
    q = np.array([[0.0, 0.0, 0.0, 1.0], [math.sqrt(0.5), 0.0, 0.0, math.sqrt(0.5)], [0.1, -0.2, 0.3, -0.9]])
    packed = sf._smallest_three(q)
    assert packed[0] == (3 << 30)
    cols = [bytes(27), bytes(3), bytes(9), bytes(9), packed.astype("<u4").tobytes(), b""]
    out = np.zeros((3, 4))
    c = [np.frombuffer(x, dtype=np.uint8) if x else np.zeros(1, np.uint8) for x in cols]
    orc.lib().orc_spz_decode(3, 3, 0, 12, *(orc._p(x) for x in c), 0, None, None, orc._p(out), None, None)
    assert np.array_equal(out[0], [0, 0, 0, 1])
    for i in (1, 2):
        assert abs(abs(np.dot(out[i], _unit(q)[i])) - 1) < 1e-5


def test_malformed_files_fail_with_the_reference_texts():
    d = syn.mixture_table(50, seed=40, sh_degree=1)
    good = sf.gzip_spz(d)
    with pytest.raises(ValueError, match="Invalid SPZ file"):
        orc.spz_unpack(b"PK\x03\x04" + bytes(40))
    with pytest.raises(ValueError, match="Invalid SPZ file"):
        orc.spz_unpack(gzip.compress(bytes(64)))
    body = gzip.decompress(good)
    with pytest.raises(ValueError, match="Unsupported SPZ version 5 or SH degree 1"):
        orc.spz_unpack(gzip.compress(body[:4] + struct.pack("<I", 5) + body[8:]))
    with pytest.raises(ValueError, match="Unsupported SPZ version 3 or SH degree 7"):
        orc.spz_unpack(gzip.compress(body[:12] + bytes([7]) + body[13:]))
    with pytest.raises(ValueError, match="ended unexpectedly"):
        orc.spz_unpack(gzip.compress(body[:-10]))
    if orc.zstd_lib() is None:
        return
    ng = sf.ngsp_spz(d)
    with pytest.raises(ValueError, match="in the NGSP container"):
        orc.spz_unpack(ng[:4] + struct.pack("<I", 3) + ng[8:])
    with pytest.raises(ValueError, match="table of contents inside the header"):
        orc.spz_unpack(ng[:16] + struct.pack("<I", 8) + ng[20:])
    with pytest.raises(ValueError, match="streams, 6 expected"):
        orc.spz_unpack(ng[:15] + bytes([5]) + ng[16:])
    with pytest.raises(ValueError, match="bytes after its last stream"):
        orc.spz_unpack(ng + b"\0")
    with pytest.raises(ValueError, match="sizes don't match its header"):
        toc = struct.unpack_from("<I", ng, 16)[0]
        orc.spz_unpack(ng[:toc + 8] + struct.pack("<I", 1) + ng[toc + 12:])
