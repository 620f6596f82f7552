"""The ray projection methods (3dgut, htgs, raygs) on the GPU against the
float64 oracle, through rdx_project_words: every head and eye word of the
reference's layout (src/render/projections.tsl.ts:5-17) and the keys, for raw
float32 / float16 tables, ext, packed and cov tables with either SH codec,
stereo, an orthographic eye, collections with rotated and uniformly scaled
objects, non-uniform and mirrored objects (through fromCov), per-object
params, and keys without cull_keys.

Both sides compute in float64 with the same operation order (the kernel's file
is compiled without multiply-add contraction), so words are bit-equal except
where a transcendental function's last-ulp difference crosses a rounding
boundary of a quantised field: at most one word in a thousand may differ, and
a drawn-eye decision may differ for a handful of splats on a threshold (keys
then differ for those splats alone). raygs' c^2 word is a float32: within one
float32 step."""
import math

import numpy as np
import pytest

import radix_b200 as rb
from radix_b200 import _abi
from oracle import oracle as orc
from radix_b200 import camera as cm
from radix_b200 import synthetic as syn
from tests import ray_words as rw
from tests.parity import cuda_table, u32
from tests.test_gpu_layouts import _tables

pytestmark = pytest.mark.gpu
METHODS = ("3dgut", "htgs", "raygs")
MAX_WORD_MISMATCH = 1e-3


def check(objects_gpu, objects_orc, cam, method, params=None, bits=32, cull_keys=True):
    gpu = rb.project_words(objects_gpu, cam, method, params, bits, cull_keys)
    ref = orc.project_rays(objects_orc, cam, method, params, bits, cull_keys)
    eyes = len(cam.eyes)
    assert tuple(gpu["words"].shape) == ref["words"].shape == (ref["keys"].shape[0], rb.method_words(method, eyes))
    r = rw.compare(u32(gpu["words"]), ref["words"], u32(gpu["keys"]), ref["keys"], method, eyes)
    print(method, r)
    assert r["drawn"] > 0
    assert r["drawn_disagreements"] <= max(2, r["rows"] * eyes // 10_000), r
    assert r["key_mismatches"] <= (r["drawn_disagreements"] if cull_keys else 0), r
    assert r["word_mismatch_share"] <= MAX_WORD_MISMATCH, r
    for e in range(eyes):
        assert r.get(f"c2_rel_{e}", 0.0) <= 1.2e-7, r
    return gpu, ref, r


@pytest.mark.parametrize("method", METHODS)
def test_raw_float32_sh3(ctx, method):
    d = syn.mixture_table(60_000, seed=41, sh_degree=3)
    d["opacities"][::9] = np.float32(1.6)  # LoD opacities: stretch and inflate
    check([rb.SplatObject(cuda_table(d))], [rb.SplatObject(rb.Table.from_dict(d))], syn.scale_camera(), method)


@pytest.mark.parametrize("method", METHODS)
def test_stereo_float16_colours(ctx, method):
    d = syn.mixture_table(40_000, seed=42, sh_degree=3, color_dtype=np.float16)
    check([rb.SplatObject(cuda_table(d))], [rb.SplatObject(rb.Table.from_dict(d))], syn.stereo_camera(), method, bits=24)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("layout,codec", [("ext", "ext"), ("ext", "packed"), ("packed", "packed")])
def test_ext_and_packed_tables(ctx, method, layout, codec):
    d = syn.mixture_table(30_000, seed=43, sh_degree=2)
    dev, hst = _tables(d, layout, codec, False)
    check([rb.SplatObject(dev)], [rb.SplatObject(hst)], syn.scale_camera(), method)


def _world(angle, scale, t):
    c, s = math.cos(angle), math.sin(angle)
    axis = np.array([1.0, 2.0, 0.5]) / math.sqrt(5.25)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    m = np.eye(4)
    m[:3, :3] = (np.eye(3) + s * K + (1 - c) * K @ K) * scale
    m[:3, 3] = t
    return m.T.reshape(16)


@pytest.mark.parametrize("method", METHODS)
def test_collection_with_transforms_and_params(ctx, method):
    d1 = syn.mixture_table(30_000, seed=44, sh_degree=3)
    d2 = syn.plain_table(20_000, seed=45)
    worlds = [_world(0.7, 1.5, (0.3, -0.2, 0.4)), _world(-0.4, 0.6, (0.0, 0.5, -1.0))]
    over = rb.SplatParams(focal_distance=3.0, aperture_tan=0.02, pre_blur_amount=0.2, max_sh_degree=1)
    objs_gpu = [rb.SplatObject(cuda_table(d1), world=worlds[0]),
                rb.SplatObject(cuda_table(d2), count=15_000, world=worlds[1], params=over)]
    objs_orc = [rb.SplatObject(rb.Table.from_dict(d1), world=worlds[0]),
                rb.SplatObject(rb.Table.from_dict(d2), count=15_000, world=worlds[1], params=over)]
    check(objs_gpu, objs_orc, syn.scale_camera(), method, bits=24)
    check(objs_gpu, objs_orc, syn.scale_camera(), method, bits=16, cull_keys=False)
    guard = rb.SplatParams(sort_guard=0.2)
    check(objs_gpu, objs_orc, syn.scale_camera(), method, guard, bits=32, cull_keys=False)


@pytest.mark.parametrize("method", METHODS)
def test_orthographic_eye(ctx, method):
    d = syn.plain_table(40_000, seed=46)
    view = cm.look_at((0.0, 0.5, 3.0), (0, 0, 0))
    proj = np.zeros((4, 4))
    proj[0, 0], proj[1, 1], proj[2, 2], proj[2, 3], proj[3, 3] = 1 / 1.6, 1 / 0.9, -1 / 50, -0.0, 1.0
    cam = rb.Camera(view, [(view, proj.T.reshape(16), True)], 1600, 900)
    check([rb.SplatObject(cuda_table(d))], [rb.SplatObject(rb.Table.from_dict(d))], cam, method)


def test_ewa_method_forwards_to_the_projection(ctx):
    d = syn.mixture_table(30_000, seed=47, sh_degree=3)
    objs = [rb.SplatObject(cuda_table(d))]
    cam = syn.scale_camera()
    w = rb.project_words(objs, cam, "ewa", sort_bits=32)
    p = rb.project_collection(objs, cam, None, 32, cull_keys=True, outputs=("words", "keys"))
    assert np.array_equal(u32(w["words"]).reshape(-1), u32(p["words"]).reshape(-1))
    assert np.array_equal(u32(w["keys"]), u32(p["keys"]))


@pytest.mark.parametrize("method", METHODS)
def test_non_uniform_and_mirrored_objects(ctx, method):
    """Object matrices that are not a rotation times a uniform scale reach the
    splat form through the covariance and fromCov's Jacobi eigen decomposition."""
    d1 = syn.mixture_table(30_000, seed=49, sh_degree=2)
    d2 = syn.plain_table(20_000, seed=50)
    stretch = _world(0.5, 1.0, (0.2, 0.0, -0.3))
    stretch[4:7] *= 1.8  # columns 1 and 2 scaled: R diag(1, 1.8, 0.6), a non-uniform scale
    stretch[8:11] *= 0.6
    mirror = _world(0.2, 1.0, (0.0, 0.1, -0.3))
    mirror[0:3] = -mirror[0:3]  # the first column negated: a mirror
    objs_gpu = [rb.SplatObject(cuda_table(d1), world=stretch), rb.SplatObject(cuda_table(d2), world=mirror)]
    objs_orc = [rb.SplatObject(rb.Table.from_dict(d1), world=stretch), rb.SplatObject(rb.Table.from_dict(d2), world=mirror)]
    check(objs_gpu, objs_orc, syn.scale_camera(), method, bits=24)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("codec", ["ext", "packed"])
def test_cov_tables(ctx, method, codec):
    d = syn.mixture_table(30_000, seed=51, sh_degree=3)
    d["opacities"][::7] = np.float32(1.5)
    dev, hst = _tables(d, "cov", codec, False)
    check([rb.SplatObject(dev)], [rb.SplatObject(hst)], syn.scale_camera(), method)
    check([rb.SplatObject(dev)], [rb.SplatObject(hst)], syn.stereo_camera(), method, bits=16)


def test_refusals(ctx):
    d = syn.mixture_table(5_000, seed=48, sh_degree=1)
    cam = syn.scale_camera()
    with pytest.raises(_abi.RadixError) as e:
        rb.project_words([rb.SplatObject(rb.Table.from_dict(d))], cam, "3dgut")  # host memory
    assert e.value.code == _abi.RDX_ERR_ARG
    assert [rb.method_words(m, e) for m in ("ewa", "3dgut", "htgs", "raygs") for e in (1, 2)] == [4, 8, 8, 10, 8, 10, 7, 10]
