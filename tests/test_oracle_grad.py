"""The oracle's analytic gradient of the projection against central finite
differences (h = 1e-4) of its own float64 forward, on seeded splats of the
Gaussian-mixture workload, mono and stereo, with the LoD and depth-of-field
branches. CPU only."""
import numpy as np
import pytest

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import synthetic as syn
from tests.grad_check import compare, finite_differences, upstream


def _analytic(d, cam, up, params=None):
    g = orc.project_backward([rb.SplatObject(rb.Table.from_dict(d))], cam, up, params)
    deg = d["sh_degree"]
    g["colors"] = g["colors"][:, :(1 + (deg + 1) ** 2 - 1) * 3]
    return g


def _check(d, cam, params=None, rel=1e-4, min_frac=0.995):
    up = upstream(d["centers"].shape[0], len(cam.eyes))
    g = _analytic(d, cam, up, params)
    fd, bad = finite_differences(d, cam, up, params=params)
    rep = compare(g, fd, bad, rel=rel)
    for k, (frac, worst, count) in rep.items():
        assert count > 0, k
        assert frac >= min_frac, (k, frac, worst, rep)
    return rep


def test_sh_basis_gradient_matches_differences():
    rng = np.random.default_rng(3)
    for _ in range(20):
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        g = orc.sh_basis_grad(v)
        for j in range(3):
            e = np.zeros(3)
            e[j] = 1e-6
            num = (orc.sh_basis(v + e) - orc.sh_basis(v - e)) / 2e-6
            np.testing.assert_allclose(g[:, j], num, rtol=1e-6, atol=1e-7)


def test_gradient_mono_sh3():
    d = syn.mixture_table(400, seed=2, sh_degree=3)
    print(_check(d, syn.scale_camera()))


def test_gradient_stereo_sh2():
    d = syn.mixture_table(300, seed=4, sh_degree=2)
    print(_check(d, syn.stereo_camera()))


def test_gradient_lod_opacity_and_depth_of_field():
    d = syn.mixture_table(300, seed=5, sh_degree=1)
    d["opacities"] = (d["opacities"] * 1.8).astype(np.float32)  # some above 1: the LoD branch
    p = rb.SplatParams(focal_distance=5.0, aperture_tan=0.002)
    print(_check(d, syn.scale_camera(), p))
    p2 = rb.SplatParams(lod_inflate=False)
    print(_check(d, syn.scale_camera(), p2))
