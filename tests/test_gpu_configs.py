"""Parity at the benchmark configurations themselves, against the float64 oracle.

* Large stereo (SH 3 stored as float16, two eyes 2064x2208, fov 100, a 64 mm
  baseline, one key per splat from the head): keys and the order bit-exact,
  every output within 1e-5 per eye, for the plain frame and for the same
  view as a graph batch.
* Batched (16 scenes of 50k-2M splats, 64 views on a sphere of radius 4,
  one CUDA graph): every view's keys, order and visible count bit-exact, its
  outputs within 1e-5.
* Differentiable (1M splats, SH 3): the gradient on 1,000 splats sampled with
  seed 2, against float64 central differences (h = 1e-4) of the oracle's
  forward on those splats; every differentiable entry within 1e-4.

The stereo semantics are the reference's: one sort from the head, eyes
projected separately (docs/xr.md:25-33); SH evaluated once from the head.
"""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from radix_b200.synthetic import Mulberry32
from tests.grad_check import compare, finite_differences, upstream
from tests.parity import TOLERANCE, compare_projection, cuda_table, host, rel_errors, u32

pytestmark = pytest.mark.gpu
NAMES = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")


def _per_eye_errors(gpu, ref):
    """Max relative error of every output, eye by eye."""
    eyes = ref["visible"].shape[0]
    errs = []
    for e in range(eyes):
        g = {k: host(gpu[k])[e:e + 1] for k in ("mean2d", "conic", "depth", "opacity", "rgb")}
        o = {k: ref[k][e:e + 1] for k in g}
        gvis = g["opacity"] > 0
        ovis = ref["visible"][e:e + 1].astype(bool)
        assert int(np.sum(gvis != ovis)) == 0, ("cull decisions differ", e)
        errs.append(rel_errors(g, o, ovis))
    return errs


def test_large_stereo_fp16_sh3_plain_and_batched(ctx):
    n = 2_000_000
    d = syn.mixture_table(n, seed=0, sh_degree=3, color_dtype=np.float16)
    cam = syn.stereo_camera()
    obj = [rb.SplatObject(cuda_table(d))]
    res = rb.frame(obj, cam, None, 32, NAMES)
    ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cam, None, 32, cull_keys=True)
    np.testing.assert_array_equal(u32(res["keys"]), ref["keys"])
    errs = _per_eye_errors(res, ref)
    print({"eye errors": errs, "drawn": [int(v.sum()) for v in ref["visible"]]})
    for e, per in enumerate(errs):
        for name, err in per.items():
            assert err < TOLERANCE, (e, name, err)
    order, visible = orc.sort(ref["keys"], n, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"]), order[:n])
    # the same view as a one-view graph batch: the same bits
    batch = rb.Batch([(obj, cam)], None, 32, NAMES)
    batch.launch()
    batch.synchronize()
    got = batch.results()
    for k in NAMES:
        np.testing.assert_array_equal(host(got[k]), host(res[k]), err_msg=k)
    np.testing.assert_array_equal(u32(got["ordering"]), u32(res["ordering"]))
    assert int(host(got["visible"])[0]) == visible
    batch.close()


def test_batched_64_views_of_16_scenes(ctx):
    counts = syn.batched_counts(16, seed=2)
    dicts = [syn.mixture_table(c, seed=100 + s, sh_degree=3) for s, c in enumerate(counts)]
    tables = [cuda_table(d) for d in dicts]
    cams = syn.sphere_cameras(64, seed=1)
    views = [([rb.SplatObject(tables[v % 16])], cams[v]) for v in range(64)]
    batch = rb.Batch(views, None, 32, NAMES)
    batch.launch()
    batch.synchronize()
    got = batch.results()
    visible = host(got["visible"]).view(np.uint32)
    first = 0
    worst = {}
    for v in range(64):
        d = dicts[v % 16]
        nv = d["centers"].shape[0]
        ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cams[v], None, 32, cull_keys=True)
        view = {k: got[k][first:first + nv] if k == "keys" else got[k][:, first:first + nv] for k in NAMES}
        r = compare_projection(view, ref)
        assert r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, (v, r)
        for name, e in r["errors"].items():
            assert e < TOLERANCE, (v, name, e)
            worst[name] = max(worst.get(name, 0.0), e)
        order, vis = orc.sort(ref["keys"], nv, 32)
        assert int(visible[v]) == vis, v
        np.testing.assert_array_equal(u32(got["ordering"][first:first + nv]), order[:nv], err_msg=f"view {v}")
        first += nv
    print({"splat_views": first, "worst": worst})
    batch.close()


def test_gradient_against_finite_differences_on_1k_sampled_splats(ctx):
    n, k = 1_000_000, 1_000
    d = syn.mixture_table(n, seed=0, sh_degree=3)
    cam = syn.scale_camera()
    up64 = {name: v.astype(np.float32).astype(np.float64) for name, v in upstream(n, 1, seed=1).items()}
    obj = [rb.SplatObject(cuda_table(d))]
    fwd = rb.project_collection(obj, cam, None, 32, "full", True, outputs=("opacity",))
    g = rb.project_backward(obj, cam, {name: torch.from_numpy(v.astype(np.float32)).cuda() for name, v in up64.items()},
                            fwd["opacity"])[0]
    # 1,000 distinct splats drawn with seed 2
    idx = np.sort(np.argsort(Mulberry32(2).uniform(n), kind="stable")[:k])
    sub = {f: (d[f][idx] if f != "sh_degree" else d[f]) for f in d}
    up_sub = {name: v[:, idx] for name, v in up64.items()}
    got = {f: host(v).astype(np.float64)[idx] for f, v in g.items()}
    got["colors"] = got["colors"].reshape(k, -1)
    fd, bad = finite_differences(sub, cam, up_sub, h=1e-4)
    rep = compare(got, fd, bad, rel=1e-4)
    print({f: {"within_1e-4": frac, "worst": worst, "entries": count, "excluded": int(bad[f].sum())}
           for f, (frac, worst, count) in rep.items()})
    for f, (frac, worst, count) in rep.items():
        assert count > 0 and frac == 1.0, (f, frac, worst, rep)


def test_all_visible_pose_draws_every_splat(ctx):
    """The camera that keeps the whole mixture box inside the culls (the pose
    that makes the projection read every splat's full row)."""
    n = 200_000
    d = syn.mixture_table(n, seed=5, sh_degree=3)
    cam = syn.all_visible_camera()
    res = rb.frame([rb.SplatObject(cuda_table(d))], cam, None, 32, NAMES)
    ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cam, None, 32, cull_keys=True)
    r = compare_projection(res, ref)
    assert r["cull_disagreements"] == 0 and r["key_mismatches"] == 0, r
    assert r["drawn"] >= 0.999 * n, r["drawn"]
    for name, e in r["errors"].items():
        assert e < TOLERANCE, (name, e)
    order, visible = orc.sort(ref["keys"], n, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"]), order[:n])
