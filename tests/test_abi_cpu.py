"""The C-ABI library without a GPU: it loads, exports every symbol the header
declares, its structs have the ctypes layout, and the host-side helpers
(params, capacities, cameras, the seeded generator) behave. No kernel runs."""
import ctypes
import math
import os
import re
import subprocess

import numpy as np
import pytest

import radix_b200 as rb
from radix_b200 import _abi
from radix_b200 import camera as cm
from radix_b200.synthetic import Mulberry32

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "radix_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rdx_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _abi.SIGNATURES, f"{name} has no ctypes signature"


def test_method_words_match_the_reference_layouts():
    """ProjectionDef.headWords + eyes * eyeWords (src/render/projections.tsl.ts:5-17; the
    reference's test table at test/gpu/renderUtils.ts:116-117), and -1 out of range."""
    head = {"ewa": 0, "3dgut": 6, "htgs": 6, "raygs": 4}
    per_eye = {"ewa": 4, "3dgut": 2, "htgs": 2, "raygs": 3}
    for name, method in rb.PROJECTION_METHODS.items():
        for eyes in (1, 2):
            assert _abi.lib().rdx_method_words(method, eyes) == head[name] + eyes * per_eye[name]
        assert _abi.lib().rdx_method_words(method, 3) == -1
    assert _abi.lib().rdx_method_words(4, 1) == -1
    with pytest.raises(ValueError):
        rb.method_words("raygs", 0)


def test_version_and_default_params():
    assert _abi.lib().rdx_version() == 1
    p = _abi.rdx_params()
    _abi.lib().rdx_params_default(ctypes.byref(p))
    d = rb.SplatParams()
    for f in d.__dataclass_fields__:
        assert getattr(p, f) == pytest.approx(float(getattr(d, f)), rel=1e-7), f


def test_struct_layouts_match_the_c_compiler(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "radix_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(rdx_table), sizeof(rdx_params),'
        ' sizeof(rdx_eye), sizeof(rdx_camera), sizeof(rdx_object), sizeof(rdx_outputs), sizeof(rdx_view),'
        ' sizeof(rdx_tune_result), offsetof(rdx_camera, width), offsetof(rdx_table, ext_sh), offsetof(rdx_view, camera),'
        ' offsetof(rdx_tune_result, cand_ms)); return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(t) for t in (_abi.rdx_table, _abi.rdx_params, _abi.rdx_eye, _abi.rdx_camera, _abi.rdx_object,
                                       _abi.rdx_outputs, _abi.rdx_view, _abi.rdx_tune_result)]
    want += [_abi.rdx_camera.width.offset, _abi.rdx_table.ext_sh.offset, _abi.rdx_view.camera.offset,
             _abi.rdx_tune_result.cand_ms.offset]
    assert got == want


def test_context_without_a_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert _abi.lib().rdx_ctx_create(0, ctypes.byref(h)) == _abi.RDX_ERR_CUDA
    assert not h.value
    with pytest.raises(rb.RadixError):
        rb.Context(0)


def test_align_capacity_and_key_constants():
    assert rb.align_capacity(0) == 4096 and rb.align_capacity(4096) == 4096 and rb.align_capacity(4097) == 8192
    assert rb.SortKeys.invalid(16) == 0xFFFF and rb.SortKeys.invalid(32) == 0xFFFFFFFF
    assert rb.SortKeys.valid_max(24) == 0xFEFFFF and rb.SortKeys.valid_max(32) == 0xFEFFFFFF


def _mulberry32_scalar(seed, n):
    """mulberry32 as scripts/check-core.ts:43-48 writes it, with JS int32 semantics."""
    out = []

    def imul(a, b):
        return ((a & 0xFFFFFFFF) * (b & 0xFFFFFFFF)) & 0xFFFFFFFF

    for _ in range(n):
        seed = (seed + 0x6D2B79F5) & 0xFFFFFFFF
        t = imul(seed ^ (seed >> 15), 1 | seed)
        t = ((t + imul(t ^ (t >> 7), 61 | t)) & 0xFFFFFFFF) ^ t
        out.append(((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296)
    return np.array(out)


def test_vectorised_mulberry32_matches_the_scalar_generator():
    r = Mulberry32(12345)
    a = r.uniform(50)
    b = r.uniform(50)
    np.testing.assert_array_equal(np.concatenate([a, b]), _mulberry32_scalar(12345, 100))


def test_perspective_and_look_at():
    p = cm.perspective(60.0, 2.0, 0.1, 100.0)
    t = math.tan(math.radians(30))
    assert p[0] == pytest.approx(1 / (t * 2)) and p[5] == pytest.approx(1 / t)
    assert p[10] == pytest.approx(-100 / 99.9) and p[11] == -1.0 and p[14] == pytest.approx(-10 / 99.9)
    v = np.asarray(cm.look_at((0, 0.5, 3), (0, 0, 0))).reshape(4, 4).T
    # the target sits on the view's -z axis
    tgt = v @ np.array([0, 0, 0, 1.0])
    assert abs(tgt[0]) < 1e-12 and abs(tgt[1]) < 1e-12 and tgt[2] < 0
    cam = rb.Camera.stereo((0, 0.5, 3), (0, 0, 0), 100, 2064, 2208, baseline=0.064)
    e0 = np.asarray(cam.eyes[0][0]).reshape(4, 4).T
    e1 = np.asarray(cam.eyes[1][0]).reshape(4, 4).T
    pos0 = np.linalg.inv(e0)[:3, 3]
    pos1 = np.linalg.inv(e1)[:3, 3]
    assert np.linalg.norm(pos1 - pos0) == pytest.approx(0.064)
