"""The bounds-checked build (RDX_CHECK): the same kernels, with every index a
kernel clamps also recorded in the device error word, which the calls report
as an error. compute-sanitizer is closed on the GPUs these tests run on; this
build checks, without faulting anything, that no launch of the sort, frame,
batch, splat-sort, pinned-table and gradient paths ever computes an index
outside its buffer. The paths run in a child process that loads
radix_b200/lib/libradix_b200_check.so (RADIX_B200_CHECK=1), and their results
are compared with the float64 oracle there."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r'''
import numpy as np, torch
import radix_b200 as rb
from radix_b200 import _abi, synthetic as syn
from oracle import oracle as orc
assert _abi.LIB_PATH.endswith("libradix_b200_check.so"), _abi.LIB_PATH
u32 = lambda t: t.cpu().numpy().view(np.uint32) if hasattr(t, "cpu") else t.view(np.uint32)
ctx = rb.Context(0)
# every digit-pass variant, in both sort forms, on sizes around the tile and sub-tile edges
for variant in range(7):
    ctx.set_sort_variant(variant)
    for count, bits in ((1, 32), (4097, 16), (70000, 24), (1_000_003, 32), (4_000_000, 32)):
        keys = (syn.Mulberry32(count + variant).uniform(count) * 2.0 ** bits).astype(np.uint64).astype(np.uint32)
        keys[::3] = rb.SortKeys.invalid(bits)
        expected, visible = orc.sort(keys, count, bits)
        order, vis = rb.SortKeys.sort(torch.from_numpy(keys.view(np.int32)).cuda(), count, bits, ctx=ctx)
        ctx.synchronize()
        assert vis == visible and np.array_equal(u32(order)[:count], expected[:count]), (variant, count, bits)
        kt, vt = torch.from_numpy(keys.view(np.int32)).cuda(), torch.arange(count, dtype=torch.int32).cuda()
        rb.RadixSort(kt, vt, ctx).sort(count, bits)
        ctx.synchronize()
        assert np.array_equal(u32(vt), expected[:count]), ("pairs", variant, count, bits)
ctx.set_sort_variant(-1)
# a tuned frame, a batch of views, the splat sorter and the gradient
d = syn.mixture_table(1_000_000, seed=3, sh_degree=3)
t = rb.Table.from_dict(d, to=lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda())
cam = syn.scale_camera()
names = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")
batch = rb.Batch([([rb.SplatObject(t)], cam)], None, 32, names, ctx=ctx)
batch.tune(reps=2)
batch.launch(); batch.synchronize()
ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], cam, None, 32, cull_keys=True)
order, visible = orc.sort(ref["keys"], ref["keys"].size, 32)
assert np.array_equal(u32(batch.results()["ordering"]), order[:ref["keys"].size])
batch.close()
views = [([rb.SplatObject(t, count=c)], v) for c, v in zip((1_000_000, 300_000, 5_000), syn.sphere_cameras(3, seed=4))]
res = rb.frame_batched(views, None, 24, names, ctx=ctx)
ctx.synchronize()
keys = u32(res["keys"])
n0 = 1_000_000
o0, v0 = orc.sort(keys[:n0], n0, 24)
assert np.array_equal(u32(res["ordering"])[:n0], o0[:n0])
sorter = rb.SplatSorter(ctx)
values, count, args = sorter.sort(res["keys"][:n0], n0, 24)
ctx.synchronize()
valid = int((keys[:n0] != rb.SortKeys.invalid(24)).sum())
assert sorter.read_count() == valid and np.array_equal(u32(values)[:valid], o0[:valid])
# a pinned host table: colour rows read in place by the staging flavour
cols = ("centers", "log_scales", "quats", "opacities", "colors")
pinned = rb.Table.raw(*(torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory() for k in cols), 3)
ref_frame = rb.frame([rb.SplatObject(t)], syn.stereo_camera(), None, 32, names, ctx=ctx)
got_frame = rb.frame([rb.SplatObject(pinned)], syn.stereo_camera(), None, 32, names, ctx=ctx)
for k in names:
    assert np.array_equal(u32(got_frame[k]), u32(ref_frame[k])), ("pinned", k)
assert np.array_equal(u32(got_frame["ordering"]), u32(ref_frame["ordering"]))
fwd = rb.project_collection([rb.SplatObject(t)], cam, None, 32, "full", True, outputs=("opacity",), ctx=ctx)
up = {k: torch.randn(fwd["opacity"].shape + ((2,) if k == "mean2d" else (3,) if k in ("conic", "rgb") else ()),
                     device="cuda") for k in ("mean2d", "conic", "opacity", "rgb")}
rb.project_backward([rb.SplatObject(t)], cam, up, fwd["opacity"], ctx=ctx)
ctx.synchronize()
print("check build ok")
'''


def test_no_launch_clamps_an_index_in_the_bounds_checked_build():
    lib = os.path.join(ROOT, "radix_b200", "lib", "libradix_b200_check.so")
    assert os.path.exists(lib), "build the checked twin: python radix_b200/build.py --check"
    env = dict(os.environ, RADIX_B200_CHECK="1", PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "check build ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
