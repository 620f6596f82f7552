"""A whole frame (projection + SH + keys + sort) against the oracle: the order
bit-exact against SortKeys.sort of the oracle's keys, at the 4M-splat SH-3
workload and at small sizes, from device and from host buffers."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests.parity import compare_projection, cuda_table, host, u32

pytestmark = pytest.mark.gpu


def _frame_check(d, cam, bits, device="cuda"):
    table = cuda_table(d) if device == "cuda" else rb.Table.from_dict(d)
    res = rb.frame([rb.SplatObject(table)], cam, None, bits, device=device)
    ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cam, None, bits, cull_keys=True)
    n = d["centers"].shape[0]
    r = compare_projection(res, ref)
    assert r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, r
    expected, visible = orc.sort(ref["keys"], n, bits)
    assert res["visible"] == visible == int(ref["visible"].any(axis=0).sum())
    np.testing.assert_array_equal(u32(res["ordering"])[:n], expected[:n])
    # size-independent properties: keys ascend along the order, ties by index
    k = ref["keys"][expected[:n]]
    assert (np.diff(k.astype(np.int64)) >= 0).all()
    return r


@pytest.mark.parametrize("bits", [16, 24, 32])
def test_frame_plain_100k(ctx, bits):
    _frame_check(syn.plain_table(100_000, seed=0), syn.plain_camera(), bits)


def test_frame_4m_sh3_bit_exact_order(ctx):
    r = _frame_check(syn.mixture_table(4_000_000, seed=0, sh_degree=3), syn.scale_camera(), 32)
    print(r)
    for name, e in r["errors"].items():
        assert e < 1e-5, (name, e)


def test_frame_from_host_buffers(ctx):
    _frame_check(syn.plain_table(30_000, seed=5), syn.plain_camera(), 24, device=None)


NAMES = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")


def _same_frame(got, ref):
    for k in NAMES:
        np.testing.assert_array_equal(host(got[k]), host(ref[k]), err_msg=k)
    np.testing.assert_array_equal(u32(got["ordering"]), u32(ref["ordering"]))
    assert got["visible"] == ref["visible"]


@pytest.mark.parametrize("eyes", [1, 2])
def test_frame_reads_pinned_host_columns_in_place(ctx, eyes):
    """A raw SH-3 table in pinned host memory. Read in place (the default), the
    kernel stages the colour rows of the splats that pass the centre culls from
    host memory and the other columns are copied in; with copies, every column
    is. Both give the device table's bits; the bytes moved are the copied
    columns plus a 192-byte row per candidate, or the whole table."""
    n = 200_000
    d = syn.mixture_table(n, seed=7, sh_degree=3)
    cam = syn.scale_camera() if eyes == 1 else syn.stereo_camera()
    cols = ("centers", "log_scales", "quats", "opacities", "colors")
    pinned = {k: torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory() for k in cols}
    dev = {k: v.cuda() for k, v in pinned.items()}

    def table(c):
        return rb.Table.raw(c["centers"], c["log_scales"], c["quats"], c["opacities"], c["colors"], 3)

    ref = rb.frame([rb.SplatObject(table(dev))], cam, None, 32, NAMES, ctx=ctx)
    size = {k: v.numel() * v.element_size() for k, v in pinned.items()}
    copied = size["centers"] + size["log_scales"] + size["opacities"] + size["quats"]
    row = 16 * 3 * 4
    try:
        for in_place in (True, False):
            ctx.set_host_reads(in_place)
            ctx.host_bytes()
            got = rb.frame([rb.SplatObject(table(pinned))], cam, None, 32, NAMES, ctx=ctx)
            moved = ctx.host_bytes()
            _same_frame(got, ref)
            if in_place:
                assert (moved - copied) % row == 0, moved
                candidates = (moved - copied) // row
                assert ref["visible"] <= candidates < n, (candidates, ref["visible"])
            else:
                assert moved == sum(size.values())
    finally:
        ctx.set_host_reads(True)


def test_in_place_rows_float16_and_a_mixed_collection(ctx):
    """Float16 SH-3 rows (96 bytes: six 16-byte pieces) read in place, and a
    collection of a pinned table and a device table of the same kind in one
    launch (the staging flavour reads both): the device tables' bits."""
    cols = ("centers", "log_scales", "quats", "opacities", "colors")
    d0 = syn.mixture_table(90_000, seed=11, sh_degree=3, color_dtype=np.float16)
    d1 = syn.mixture_table(70_000, seed=12, sh_degree=3, color_dtype=np.float16)
    pin0 = {k: torch.from_numpy(np.ascontiguousarray(d0[k])).pin_memory() for k in cols}
    dev0 = {k: v.cuda() for k, v in pin0.items()}
    dev1 = {k: torch.from_numpy(np.ascontiguousarray(d1[k])).cuda() for k in cols}

    def table(c):
        return rb.Table.raw(*(c[k] for k in cols), 3)

    cam = syn.scale_camera()
    ref = rb.frame([rb.SplatObject(table(dev0)), rb.SplatObject(table(dev1))], cam, None, 32, NAMES, ctx=ctx)
    ctx.host_bytes()
    got = rb.frame([rb.SplatObject(table(pin0)), rb.SplatObject(table(dev1))], cam, None, 32, NAMES, ctx=ctx)
    moved = ctx.host_bytes()
    _same_frame(got, ref)
    copied = sum(pin0[k].numel() * pin0[k].element_size() for k in ("centers", "log_scales", "quats", "opacities"))
    assert moved > copied and (moved - copied) % 96 == 0 and (moved - copied) // 96 < 90_000


def test_in_place_rows_in_batched_frames_and_projections(ctx):
    """The other calls that stage tables: a batched frame of three views of one
    pinned table (the rows are read once per view) and projections with keys
    only (no candidate reads a row) or with every output: the device table's bits."""
    cols = ("centers", "log_scales", "quats", "opacities", "colors")
    d = syn.mixture_table(80_000, seed=13, sh_degree=3)
    pinned = {k: torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory() for k in cols}
    dev = {k: v.cuda() for k, v in pinned.items()}
    host_t = rb.Table.raw(*(pinned[k] for k in cols), 3)
    dev_t = rb.Table.raw(*(dev[k] for k in cols), 3)
    cams = syn.sphere_cameras(3, seed=14)
    ref = rb.frame_batched([([rb.SplatObject(dev_t)], c) for c in cams], None, 32, NAMES, ctx=ctx)
    got = rb.frame_batched([([rb.SplatObject(host_t)], c) for c in cams], None, 32, NAMES, ctx=ctx)
    for k in NAMES:
        np.testing.assert_array_equal(host(got[k]), host(ref[k]), err_msg=k)
    np.testing.assert_array_equal(u32(got["ordering"]), u32(ref["ordering"]))
    np.testing.assert_array_equal(host(got["visible"]), host(ref["visible"]))
    cam = syn.scale_camera()
    for pass_ in ("keys", "full"):
        a = rb.project_collection([rb.SplatObject(dev_t)], cam, None, 32, pass_, True, NAMES, ctx=ctx)
        ctx.host_bytes()
        b = rb.project_collection([rb.SplatObject(host_t)], cam, None, 32, pass_, True, NAMES, ctx=ctx)
        moved = ctx.host_bytes()
        for k in a:
            np.testing.assert_array_equal(host(b[k]), host(a[k]), err_msg=f"{pass_} {k}")
        copied = sum(pinned[k].numel() * pinned[k].element_size() for k in ("centers", "log_scales", "quats", "opacities"))
        assert moved == copied if pass_ == "keys" else moved > copied


def test_pinned_ext_table_and_guarded_raw_table_are_copied(ctx):
    """Tables whose rows no kernel flavour stages are copied in whole: an ext
    table whose SH texel channels are pinned and whose extA/extB words are
    pageable, and a pinned raw SH-3 table under a sort guard. The device
    tables' bits either way."""
    d = syn.mixture_table(60_000, seed=9, sh_degree=3)
    a, b, sh = orc.encode_ext(d)
    dev = rb.Table.ext(torch.from_numpy(a.view(np.int32)).cuda(), torch.from_numpy(b.view(np.int32)).cuda(),
                       [torch.from_numpy(c.view(np.int32)).cuda() for c in sh], 3)
    pinned_sh = [torch.from_numpy(np.ascontiguousarray(c.view(np.int32))).pin_memory() for c in sh]
    mixed = rb.Table.ext(a, b, pinned_sh, 3)
    cam = syn.scale_camera()
    ref = rb.frame([rb.SplatObject(dev)], cam, None, 32, NAMES, ctx=ctx)
    ctx.host_bytes()
    got = rb.frame([rb.SplatObject(mixed)], cam, None, 32, NAMES, ctx=ctx)
    moved = ctx.host_bytes()
    _same_frame(got, ref)
    assert moved == a.nbytes + b.nbytes + sum(c.nbytes for c in sh)
    cols = ("centers", "log_scales", "quats", "opacities", "colors")
    pinned = {k: torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory() for k in cols}
    raw = rb.Table.raw(*(pinned[k] for k in cols), 3)
    raw_dev = rb.Table.raw(*(pinned[k].cuda() for k in cols), 3)
    params = rb.SplatParams(sort_guard=1.5)
    ref = rb.frame([rb.SplatObject(raw_dev)], cam, params, 32, NAMES, ctx=ctx)
    ctx.host_bytes()
    got = rb.frame([rb.SplatObject(raw)], cam, params, 32, NAMES, ctx=ctx)
    assert ctx.host_bytes() == sum(v.numel() * v.element_size() for v in pinned.values())
    _same_frame(got, ref)


def test_frame_empty_collection(ctx):
    d = syn.plain_table(10, seed=1)
    res = rb.frame([rb.SplatObject(cuda_table(d), count=0)], syn.plain_camera(), None, 32)
    assert res["visible"] == 0
