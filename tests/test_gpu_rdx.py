"""RDX files decoded on the GPU (payloads inflated on the host, bytes
transposed back on the device) against the oracle's reader: every channel
byte-exact, into device or host arrays, over chunks with a ragged last one;
the reference's error texts; and tables over a file's splat bundles
(extSplats, covSplats, packedSplats with its encoding; per-splat SH in either
codec) projected as the oracle projects the same words."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests import rdx_fixtures as rf
from tests.parity import TOLERANCE, compare_projection, host, u32

pytestmark = pytest.mark.gpu
ALL = ("mean2d", "conic", "depth", "opacity", "rgb", "radii", "words", "keys")


def _mixed(n, seed=0):
    rng = np.random.default_rng(seed)
    return {
        "extSplats": ({"extA": "uint32x4", "extB": "uint32x4"}, {},
                      {"extA": rng.integers(0, 2**32, (n, 4), dtype=np.uint32),
                       "extB": rng.integers(0, 2**32, (n, 4), dtype=np.uint32)}),
        "misc": ({"h": "float16x3", "b": "uint8", "f": "float32x2"}, {"note": "x"},
                 {"h": rng.normal(size=(n, 3)).astype(np.float16), "b": rng.integers(0, 256, n, dtype=np.uint8),
                  "f": rng.normal(size=(n, 2)).astype(np.float32)}),
    }


@pytest.mark.parametrize("device", ["cuda", "cpu"])
def test_channels_byte_exact(ctx, device):
    n = 150_000
    raw = rf.rdx_file(_mixed(n), n, 65536)
    info, ch = rb.decode_rdxfile(raw, device=device)
    assert info["count"] == n and info["chunks"] == 3 and info["chunk_size"] == 65536
    assert [c[:3] for c in info["channels"]] == [("extSplats", "extA", "uint32x4"), ("extSplats", "extB", "uint32x4"),
                                                 ("misc", "h", "float16x3"), ("misc", "b", "uint8"),
                                                 ("misc", "f", "float32x2")]
    header, ref = orc.rdxfile_read(raw)
    assert info["header"] == header
    for name in ref:
        for label in ref[name]:
            np.testing.assert_array_equal(host(ch[name][label]), ref[name][label], err_msg=f"{name}.{label}")


def test_ragged_last_chunk(ctx):
    # 70001 rows: the first chunk's 16-byte channels go four elements a thread, the
    # last chunk's 4465 rows (not a multiple of 4) one element a thread, in one launch
    n = 70_001
    raw = rf.rdx_file(_mixed(n, seed=3), n, 65536)
    _, ch = rb.decode_rdxfile(raw)
    _, ref = orc.rdxfile_read(raw)
    for name in ref:
        for label in ref[name]:
            np.testing.assert_array_equal(host(ch[name][label]), ref[name][label], err_msg=f"{name}.{label}")


def test_errors_carry_the_reference_texts(ctx):
    raw = rf.rdx_file(_mixed(5000), 5000, 4096)
    with pytest.raises(rb.RadixError, match="Not an RDX piece of the expected type"):
        rb.rdxfile_info(b"RDXC" + raw[4:])
    with pytest.raises(rb.RadixError, match="ended unexpectedly"):
        rb.decode_rdxfile(raw[:len(raw) - 100])
    with pytest.raises(rb.RadixError, match="host memory"):
        rb.decode_rdxfile(torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda())
    bad = raw.replace(b'"uint8"', b'"uint9"', 1)
    with pytest.raises(rb.RadixError, match='Invalid array format "uint9"'):
        rb.rdxfile_info(bad)
    info, _ = rb.decode_rdxfile(raw)  # the context still works
    assert info["count"] == 5000


def _splat_file(d, layout, codec, encoding=rb.Table.PACKED_ENCODING):
    n = d["centers"].shape[0]
    deg = d["sh_degree"]
    bundles = {}
    if layout == "packed":
        enc = dict(zip(("rgbMin", "rgbMax", "lnScaleMin", "lnScaleMax"), encoding))
        bundles["packedSplats"] = ({"packed": "uint32x4"}, {"encoding": enc}, {"packed": orc.encode_packed(d, encoding)})
    elif layout == "cov":
        a, b = orc.encode_cov(d)
        bundles["covSplats"] = ({"covA": "uint32x4", "covB": "uint32x4"}, {}, {"covA": a, "covB": b})
    else:
        a, b = orc.encode_ext(d)[:2]
        bundles["extSplats"] = ({"extA": "uint32x4", "extB": "uint32x4"}, {}, {"extA": a, "extB": b})
    host_sh = ()
    if deg:
        host_sh = orc.sh_channels(orc.encode_sh(d, codec))
        labels = [f"{codec}Sh{chr(65 + i)}" for i in range(len(host_sh))]
        bundles[f"{codec}Sh"] = ({lb: "uint32x4" for lb in labels}, {"codec": codec, "degree": deg},
                                 dict(zip(labels, host_sh)))
    raw = rf.rdx_file(bundles, n, 65536)
    if layout == "packed":
        ref_table = rb.Table.packed(bundles["packedSplats"][2]["packed"], encoding, host_sh, deg, codec)
    elif layout == "cov":
        ref_table = rb.Table.cov(a, b, host_sh, deg, codec)
    else:
        ref_table = rb.Table.ext(a, b, host_sh, deg, codec)
    return raw, ref_table


@pytest.mark.parametrize("layout,codec", [("ext", "ext"), ("packed", "packed"), ("cov", "ext")])
def test_tables_over_splat_bundles(ctx, layout, codec):
    d = syn.mixture_table(100_000, seed=7, sh_degree=3)
    enc = (-0.1, 1.2, -11.0, 3.0)
    raw, ref_table = _splat_file(d, layout, codec, enc)
    table, _ = rb.rdxfile_table(raw)
    cam = syn.scale_camera()
    gpu = rb.project_collection([rb.SplatObject(table)], cam, None, 32, cull_keys=True, outputs=ALL)
    ref = orc.project([rb.SplatObject(ref_table)], cam, None, 32, True)
    r = compare_projection(gpu, ref)
    assert r["drawn"] > 0 and r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, r
    for name, e in r["errors"].items():
        assert e < TOLERANCE, (name, e, r)


def test_decoded_file_drawn_by_a_frame(ctx):
    d = syn.mixture_table(120_000, seed=9, sh_degree=2)
    raw, ref_table = _splat_file(d, "ext", "ext")
    table, _ = rb.rdxfile_table(raw)
    cam = syn.scale_camera()
    res = rb.frame([rb.SplatObject(table)], cam, None, 32)
    o = orc.project([rb.SplatObject(ref_table)], cam, None, 32, cull_keys=True)
    n = d["centers"].shape[0]
    expected, visible = orc.sort(o["keys"], n, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"])[:n], expected[:n])


@pytest.mark.parametrize("codec", ["ext", "packed"])
def test_palette_files(ctx, codec):
    """Splats with an shLabel bundle and their ShPalette in its own RDX file."""
    d = syn.mixture_table(60_000, seed=12, sh_degree=3)
    n, deg = d["centers"].shape[0], 3
    words = orc.encode_sh(d, codec)
    size = 211
    stride = 1 << (words.shape[1] // 4 - 1).bit_length()
    labels = (np.arange(n) * 7 % size).astype(np.uint16)
    entries = orc.sh_palette(np.ascontiguousarray(words[:size]), stride)
    a, b = orc.encode_ext(d)[:2]
    splats = rf.rdx_file({"extSplats": ({"extA": "uint32x4", "extB": "uint32x4"}, {}, {"extA": a, "extB": b}),
                          "shLabel": ({"label": "uint16"}, {}, {"label": labels})}, n, 65536)
    pal = rf.rdx_file({"shPalette": ({"shEntries": "uint32x4"},
                                     {"codec": codec, "degree": deg, "size": size, "stride": stride},
                                     {"shEntries": entries})}, entries.shape[0], 4096)
    table, _ = rb.rdxfile_table(splats, palette=pal)
    ref_table = rb.Table.ext(a, b, (), deg, codec, palette=(entries, labels, stride))
    cam = syn.scale_camera()
    gpu = rb.project_collection([rb.SplatObject(table)], cam, None, 32, cull_keys=True, outputs=ALL)
    ref = orc.project([rb.SplatObject(ref_table)], cam, None, 32, True)
    r = compare_projection(gpu, ref)
    assert r["drawn"] > 0 and r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, r
    for name, e in r["errors"].items():
        assert e < TOLERANCE, (name, e, r)


def test_header_json_of_every_kind(ctx):
    """The header's JSON reader: nested objects and arrays, numbers with
    exponents, booleans, null, escapes and surrogate pairs, key order kept."""
    meta = {"scene": "café \U0001F600 \"quoted\" \\ / \t", "list": [1, -2.5e3, 0.125, True, False, None],
            "nested": {"z": {"y": []}, "a": {}}}
    # names that reach the library's own reader escaped: a BMP character, a surrogate pair, a quote
    bundle, label = "b\u00e9\u2603", 'x"\U0001F600'
    raw = rf.rdx_file({bundle: ({label: "uint16x2"}, {"k": [1, {"m": "☃"}]},
                                {label: np.arange(8, dtype=np.uint16).reshape(4, 2)})}, 4, 4096, meta=meta)
    assert b"\\u2603" in raw and b"\\ud83d\\ude00" in raw and b'x\\"' in raw
    info = rb.rdxfile_info(raw)
    assert info["header"]["meta"] == meta
    assert list(info["header"]["meta"]["nested"].keys()) == ["z", "a"]
    assert info["channels"] == [(bundle, label, "uint16x2", 4)]
    _, ch = rb.decode_rdxfile(raw)
    np.testing.assert_array_equal(host(ch[bundle][label]).view(np.uint16).reshape(4, 2), np.arange(8).reshape(4, 2))
