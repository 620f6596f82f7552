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


def test_frame_empty_collection(ctx):
    d = syn.plain_table(10, seed=1)
    res = rb.frame([rb.SplatObject(cuda_table(d), count=0)], syn.plain_camera(), None, 32)
    assert res["visible"] == 0
