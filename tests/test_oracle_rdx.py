"""The RDX reader of the oracle (oracle.py rdxfile_read, restating
src/core/rdx.ts:62-205) against files written here (tests/rdx_fixtures.py):
channels of several formats round-trip byte for byte through chunks of
4096-multiple rows with a ragged last chunk, and malformed files fail with
the reference's texts."""
import gzip
import json
import struct

import numpy as np
import pytest

from oracle import oracle as orc
from tests import rdx_fixtures as rf


def _bundles(n, seed=0):
    rng = np.random.default_rng(seed)
    return {
        "extSplats": ({"extA": "uint32x4", "extB": "uint32x4"}, {},
                      {"extA": rng.integers(0, 2**32, (n, 4), dtype=np.uint32),
                       "extB": rng.integers(0, 2**32, (n, 4), dtype=np.uint32)}),
        "misc": ({"h": "float16x3", "b": "uint8", "f": "float32x2"}, {"note": 'ünïcode "quoted"'},
                 {"h": rng.normal(size=(n, 3)).astype(np.float16), "b": rng.integers(0, 256, n, dtype=np.uint8),
                  "f": rng.normal(size=(n, 2)).astype(np.float32)}),
    }


@pytest.mark.parametrize("n,chunk", [(10_000, 4096), (8192, 8192), (1, 65536), (0, 4096)])
def test_round_trip(n, chunk):
    b = _bundles(n)
    raw = rf.rdx_file(b, n, chunk, meta={"scene": "test"})
    header, out = orc.rdxfile_read(raw)
    assert header["count"] == n and header["chunkSize"] == chunk and header["meta"] == {"scene": "test"}
    assert len(header["chunks"]) == -(-n // chunk)
    for name, (channels, _, data) in b.items():
        for label, fmt in channels.items():
            want = np.ascontiguousarray(data[label]).view(np.uint8).reshape(n, rf.element_bytes(fmt))
            np.testing.assert_array_equal(out[name][label], want)


def test_malformed_files():
    b = _bundles(5000)
    raw = rf.rdx_file(b, 5000, 4096)
    with pytest.raises(ValueError, match="Not an RDX piece of the expected type"):
        orc.rdxfile_read(b"RDXC" + raw[4:])
    meta_len = struct.unpack_from("<I", raw, 4)[0]
    header = json.loads(raw[16:16 + meta_len])
    header["version"] = 2
    text = json.dumps(header, separators=(",", ":")).encode()
    assert len(text) == meta_len
    with pytest.raises(ValueError, match="RDX version 2 is not 1"):
        orc.rdxfile_read(raw[:16] + text + raw[16 + meta_len:])
    # a chunk whose payload holds the wrong number of bytes
    bad = dict(b)
    channels, bmeta, data = bad["misc"]
    bad["misc"] = ({**channels}, bmeta, data)
    short = rf.rdx_file(bad, 5000, 4096)
    hdr_len = orc._rdx_container(short, 0, orc.RDX_HEADER_MAGIC)[2]
    meta, payloads, _ = orc._rdx_container(short, hdr_len, orc.RDX_CHUNK_MAGIC)
    payloads[-1] = gzip.compress(bytes(10), mtime=0)
    chunk0 = rf.container(rf.CHUNK_MAGIC, meta, payloads)
    h = json.loads(short[16:16 + struct.unpack_from("<I", short, 4)[0]])
    rest = short[hdr_len + h["chunks"][0]:]
    h["chunks"][0] = len(chunk0)
    rebuilt = rf.container(rf.HEADER_MAGIC, h, []) + chunk0 + rest
    with pytest.raises(ValueError, match=r"Chunk at 0: misc\.f holds 10 bytes, expected 32768"):
        orc.rdxfile_read(rebuilt)
