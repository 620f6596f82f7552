"""Batched frames (many views of many collections) against one frame per view
and against the oracle, and the CUDA-graph batch against the direct call,
including camera updates between replays."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests.parity import compare_projection, cuda_table, host, u32

pytestmark = pytest.mark.gpu

NAMES = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")


def _scenes(counts, degree=3):
    return [syn.mixture_table(n, seed=10 + s, sh_degree=degree) for s, n in enumerate(counts)]


def _views(tables, cams, assign):
    return [([rb.SplatObject(tables[assign[v]])], cams[v]) for v in range(len(cams))]


def _rows(views):
    first, off = [], 0
    for objects, _ in views:
        first.append(off)
        off += sum(o.count for o in objects)
    return first, off


def _split(res, views, v):
    """View v's slice of a batched result, shaped like a single frame's."""
    first, n = _rows(views)
    nv = sum(o.count for o in views[v][0])
    out = {}
    for k in NAMES:
        a = res[k]
        out[k] = a[first[v]:first[v] + nv] if k == "keys" else a[:, first[v]:first[v] + nv]
    out["ordering"] = res["ordering"][first[v]:first[v] + nv]
    out["visible"] = int(host(res["visible"]).view(np.uint32)[v])
    return out


def _same(a, b):
    for k in NAMES:
        np.testing.assert_array_equal(host(a[k]), host(b[k]), err_msg=k)
    np.testing.assert_array_equal(u32(a["ordering"]), u32(b["ordering"]))
    assert a["visible"] == b["visible"]


@pytest.mark.parametrize("bits", [24, 32])
def test_batched_equals_one_frame_per_view(ctx, bits):
    dicts = _scenes([20_000, 65_000, 3_000])
    tables = [cuda_table(d) for d in dicts]
    cams = syn.sphere_cameras(7, seed=3)
    assign = [0, 1, 2, 0, 1, 2, 1]
    views = _views(tables, cams, assign)
    res = rb.frame_batched(views, None, bits, NAMES)
    for v, (objects, cam) in enumerate(views):
        single = rb.frame(objects, cam, None, bits, NAMES)
        _same(_split(res, views, v), single)


def test_batched_against_the_oracle(ctx):
    dicts = _scenes([30_000, 12_000], degree=2)
    tables = [cuda_table(d) for d in dicts]
    cams = syn.sphere_cameras(3, seed=4)
    assign = [0, 1, 0]
    views = _views(tables, cams, assign)
    res = rb.frame_batched(views, None, 32, NAMES)
    for v in range(3):
        got = _split(res, views, v)
        d = dicts[assign[v]]
        ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cams[v], None, 32, cull_keys=True)
        r = compare_projection(got, ref)
        assert r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, r
        for name, e in r["errors"].items():
            assert e < 1e-5, (v, name, e)
        n = d["centers"].shape[0]
        expected, visible = orc.sort(ref["keys"], n, 32)
        assert got["visible"] == visible
        np.testing.assert_array_equal(u32(got["ordering"]), expected[:n])


def test_batch_with_an_empty_view_and_a_collection(ctx):
    dicts = _scenes([8_000, 5_000], degree=1)
    tables = [cuda_table(d) for d in dicts]
    cams = syn.sphere_cameras(3, seed=5)
    views = [([rb.SplatObject(tables[0]), rb.SplatObject(tables[1])], cams[0]),
             ([rb.SplatObject(tables[1], count=0)], cams[1]),
             ([rb.SplatObject(tables[1], count=4_000)], cams[2])]
    res = rb.frame_batched(views, None, 24, NAMES)
    for v, (objects, cam) in enumerate(views):
        single = rb.frame(objects, cam, None, 24, NAMES)
        _same(_split(res, views, v), single)


def test_graph_batch_replays_and_updates(ctx):
    dicts = _scenes([40_000, 9_000, 100_000])
    tables = [cuda_table(d) for d in dicts]
    cams = syn.sphere_cameras(6, seed=6)
    assign = [0, 1, 2, 2, 1, 0]
    views = _views(tables, cams, assign)
    batch = rb.Batch(views, None, 32, NAMES)
    assert batch.launches() >= 7  # projection, counting, partition (and visible counts), 4 digit passes: one graph
    direct = rb.frame_batched(views, None, 32, NAMES)
    for _ in range(3):  # replays: fresh lookback epochs, cleared histograms
        batch.launch()
        batch.synchronize()
        got = batch.results()
        for v in range(len(views)):
            _same(_split(got, views, v), _split(direct, views, v))
    # new cameras without a new capture
    cams2 = syn.sphere_cameras(6, seed=7)
    views2 = _views(tables, cams2, assign)
    batch.update(views2)
    batch.launch()
    batch.synchronize()
    direct2 = rb.frame_batched(views2, None, 32, NAMES)
    got = batch.results()
    for v in range(len(views2)):
        _same(_split(got, views2, v), _split(direct2, views2, v))
    batch.close()


def test_graph_batch_rejects_host_memory_and_changed_views(ctx):
    d = syn.plain_table(1_000, seed=2)
    cams = syn.sphere_cameras(2, seed=8)
    with pytest.raises(rb.RadixError):
        rb.Batch([([rb.SplatObject(rb.Table.from_dict(d))], cams[0])], None, 32, NAMES)
    t = cuda_table(d)
    batch = rb.Batch([([rb.SplatObject(t)], cams[0])], None, 32, NAMES)
    with pytest.raises(rb.RadixError):
        batch.update([([rb.SplatObject(t, count=500)], cams[0])])
    with pytest.raises(rb.RadixError):
        batch.update([([rb.SplatObject(t)], cams[0]), ([rb.SplatObject(t)], cams[1])])
    batch.close()
