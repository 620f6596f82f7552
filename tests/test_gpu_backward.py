"""The CUDA gradient of the projection against the float64 oracle's analytic
gradient and against central finite differences (h = 1e-4) of the oracle's
forward: mono and stereo, float32 and float16 colours, collections with
object transforms, the LoD and depth-of-field branches, and the 1M-splat
workload."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests.grad_check import compare, finite_differences, upstream
from tests.parity import FLOOR, TOLERANCE, cuda_table, host

pytestmark = pytest.mark.gpu
FIELDS = ("centers", "log_scales", "quats", "opacities", "colors")


def _run(dicts, camera, params=None, worlds=None, seed=1):
    """CUDA and oracle gradients of one collection, with the same float32 upstream."""
    objs_gpu = [rb.SplatObject(cuda_table(d), world=None if worlds is None else worlds[i]) for i, d in enumerate(dicts)]
    objs_orc = [rb.SplatObject(rb.Table.from_dict(d), world=None if worlds is None else worlds[i])
                for i, d in enumerate(dicts)]
    n = sum(d["centers"].shape[0] for d in dicts)
    E = len(camera.eyes)
    up = {k: v.astype(np.float32) for k, v in upstream(n, E, seed).items()}
    fwd = rb.project_collection(objs_gpu, camera, params, 32, "full", True, outputs=("opacity",))
    got = rb.project_backward(objs_gpu, camera, {k: torch.from_numpy(v).cuda() for k, v in up.items()},
                              fwd["opacity"], params)
    ref = orc.project_backward(objs_orc, camera, {k: v.astype(np.float64) for k, v in up.items()}, params)
    return got, ref, dicts


def _compare(got, ref, dicts, tol=TOLERANCE):
    """Max relative error per field (floor: FLOOR x max|ref| of the field)."""
    errs = {}
    off = 0
    for g, d in zip(got, dicts):
        n = d["centers"].shape[0]
        ncol = (d["sh_degree"] + 1) ** 2 * 3
        for f in FIELDS:
            r = ref[f][off:off + n]
            if f == "colors":
                r = r[:, :ncol]
            a = host(g[f]).reshape(r.shape).astype(np.float64)
            scale = np.maximum(np.abs(r), FLOOR * max(np.abs(r).max(), 1e-30))
            errs[f] = max(errs.get(f, 0.0), float((np.abs(a - r) / scale).max()))
        off += n
    for f, e in errs.items():
        assert e < tol, (f, e, errs)
    return errs


def test_backward_mono_sh3(ctx):
    print(_compare(*_run([syn.mixture_table(20_000, seed=2, sh_degree=3)], syn.scale_camera())))


def test_backward_stereo_f16_sh2(ctx):
    d = syn.mixture_table(10_000, seed=3, sh_degree=2, color_dtype=np.float16)
    print(_compare(*_run([d], syn.stereo_camera())))


def _lod_collection():
    a = syn.mixture_table(6_000, seed=4, sh_degree=1)
    a["opacities"] = (a["opacities"] * 1.8).astype(np.float32)  # some above 1: the LoD branch
    b = syn.mixture_table(4_000, seed=5, sh_degree=1)
    t = np.eye(4)
    t[3, :3] = (0.5, -0.3, 0.2)  # a translation (column-major: elements 12-14)
    return [a, b], [None, t.reshape(16)]


def test_backward_collection_with_lod_opacity(ctx):
    dicts, worlds = _lod_collection()
    print(_compare(*_run(dicts, syn.scale_camera(), None, worlds)))
    print(_compare(*_run(dicts, syn.scale_camera(), rb.SplatParams(lod_inflate=False), worlds)))


def test_backward_depth_of_field(ctx):
    dicts, worlds = _lod_collection()
    p = rb.SplatParams(focal_distance=5.0, aperture_tan=0.002)
    print(_compare(*_run(dicts, syn.scale_camera(), p, worlds)))


def test_backward_sh0_without_clamp(ctx):
    print(_compare(*_run([syn.plain_table(20_000, seed=6)], syn.plain_camera())))


def test_backward_against_finite_differences(ctx):
    d = syn.mixture_table(300, seed=2, sh_degree=3)
    cam = syn.scale_camera()
    up = {k: v.astype(np.float32).astype(np.float64) for k, v in upstream(300, 1).items()}
    obj = [rb.SplatObject(cuda_table(d))]
    fwd = rb.project_collection(obj, cam, None, 32, "full", True, outputs=("opacity",))
    g = rb.project_backward(obj, cam, {k: torch.from_numpy(v.astype(np.float32)).cuda() for k, v in up.items()},
                            fwd["opacity"])[0]
    got = {k: host(v).astype(np.float64) for k, v in g.items()}
    got["colors"] = got["colors"].reshape(300, -1)
    fd, bad = finite_differences(d, cam, up)
    rep = compare(got, fd, bad, rel=1e-4)
    for k, (frac, worst, count) in rep.items():
        assert count > 0 and frac >= 0.995, (k, frac, worst, rep)
    print(rep)


def test_backward_1m_workload(ctx):
    d = syn.mixture_table(1_000_000, seed=0, sh_degree=3)
    print(_compare(*_run([d], syn.scale_camera())))


def test_backward_rejects_ext_tables(ctx):
    d = syn.mixture_table(100, seed=1, sh_degree=1)
    a, b, sh = orc.encode_ext(d)
    t = rb.Table.ext(*(torch.from_numpy(x.view(np.int32)).cuda() for x in (a, b)),
                     [torch.from_numpy(x.view(np.int32)).cuda() for x in sh], sh_degree=1)
    obj = [rb.SplatObject(t)]
    op = torch.zeros(100, device="cuda")
    with pytest.raises(rb.RadixError):
        rb.project_backward(obj, syn.scale_camera(), {}, op,
                            grads=[{"centers": torch.empty((100, 3), device="cuda")}])
