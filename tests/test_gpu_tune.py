"""The autotuner: it times projection block sizes and digit-pass variants on
the caller's own buffers, keeps the fastest (never slower than the defaults,
its first candidate), re-captures a batch's graph with it, and the results
stay bit-exact against the oracle (the reference's keysPerThread knob,
src/wgpu/WgpuRadixSort.ts:80-91, is chosen by hand)."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests.parity import compare_projection, cuda_table, host, u32

pytestmark = pytest.mark.gpu
NAMES = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")


def _check_tuning(r, multi_view):
    assert r["candidates"][0]["sort_variant"] == 0 and r["candidates"][0]["project_warps"] == 4
    assert r["tuned_ms"] <= r["default_ms"]
    assert r["tuned_ms"] == min(c["ms"] for c in r["candidates"])
    variants = {c["sort_variant"] for c in r["candidates"]}
    assert {0, 4, 5} <= variants
    if multi_view:
        assert not variants & {1, 2, 3}  # cooperative passes sort one segment only
    else:
        assert {1, 2, 3} <= variants
    assert {c["project_warps"] for c in r["candidates"]} >= {2, 4, 8}


def test_tuned_one_view_batch_matches_the_oracle():
    ctx = rb.Context(0)
    d = syn.mixture_table(300_000, seed=21, sh_degree=3)
    cam = syn.scale_camera()
    batch = rb.Batch([([rb.SplatObject(cuda_table(d))], cam)], None, 32, NAMES, ctx=ctx)
    r = batch.tune(reps=3)
    print(r)
    _check_tuning(r, False)
    batch.launch()
    batch.synchronize()
    got = batch.results()
    ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cam, None, 32, cull_keys=True)
    rep = compare_projection({k: got[k] for k in NAMES}, ref)
    assert rep["cull_disagreements"] == 0 and rep["key_mismatches"] == 0, rep
    assert max(rep["errors"].values()) < 1e-5
    order, visible = orc.sort(ref["keys"], ref["keys"].size, 32)
    assert int(host(got["visible"])[0]) == visible
    np.testing.assert_array_equal(u32(got["ordering"]), order[:ref["keys"].size])
    # rb.frame of the same shape takes the tuned choice from the context
    res = rb.frame([rb.SplatObject(cuda_table(d))], cam, None, 32, NAMES, ctx=ctx)
    np.testing.assert_array_equal(u32(res["ordering"]), order[:ref["keys"].size])
    batch.close()
    ctx.close()


def test_tuned_multi_view_batch_matches_direct_frames():
    ctx = rb.Context(0)
    dicts = [syn.mixture_table(n, seed=30 + i, sh_degree=2) for i, n in enumerate((50_000, 120_000))]
    tables = [cuda_table(d) for d in dicts]
    cams = syn.sphere_cameras(4, seed=9)
    views = [([rb.SplatObject(tables[v % 2])], cams[v]) for v in range(4)]
    batch = rb.Batch(views, None, 24, NAMES, ctx=ctx)
    r = batch.tune(reps=3)
    print(r)
    _check_tuning(r, True)
    batch.launch()
    batch.synchronize()
    got = batch.results()
    direct = rb.frame_batched(views, None, 24, NAMES)
    for k in NAMES:
        np.testing.assert_array_equal(host(got[k]), host(direct[k]), err_msg=k)
    np.testing.assert_array_equal(u32(got["ordering"]), u32(direct["ordering"]))
    batch.close()
    ctx.close()


@pytest.mark.parametrize("count", [5_000, 300_000, 2_000_000])
def test_tuned_sort_matches_the_oracle(count):
    ctx = rb.Context(0)
    keys = (syn.Mulberry32(count).uniform(count) * 2.0 ** 32).astype(np.uint64).astype(np.uint32)
    keys[::4] = 0xFFFFFFFF
    kt = torch.from_numpy(keys.view(np.int32)).cuda()
    r = ctx.tune_sort(kt, count, 32, reps=3)
    print(r)
    assert r["tuned_ms"] <= r["default_ms"]
    assert r["candidates"][0]["sort_variant"] == 0
    np.testing.assert_array_equal(u32(kt), keys)  # the keys are read, not changed
    order, vis = rb.SortKeys.sort(kt, count, 32, ctx=ctx)
    expected, visible = orc.sort(keys, count, 32)
    assert vis == visible
    np.testing.assert_array_equal(u32(order)[:count], expected[:count])
    ctx.close()
