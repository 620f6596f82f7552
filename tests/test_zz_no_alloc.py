"""rdx_sort_noalloc against rdx_sort and the oracle, through the C ABI.

rdx_sort_noalloc serves callers that may not allocate GPU memory (hosts that
own the device memory budget, frame loops that cannot afford an allocation's
synchronisation): its scratch is a fixed array inside the library. Calls in a
row must each give rdx_sort's order and visible count - each one finds the
array as the one before left it, whatever its size, key width and digit-pass
tile size. This file is collected last so that a run stopping at the first
failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import _abi
from radix_b200.synthetic import Mulberry32

pytestmark = pytest.mark.gpu
MAX_KEYS = 1 << 20


def _keys(n, bits, seed, invalid_every=0):
    k = (Mulberry32(seed).uniform(n) * 2.0 ** bits).astype(np.uint64).astype(np.uint32)
    if invalid_every:
        k[::invalid_every] = rb.SortKeys.invalid(bits)
    return k


def _noalloc(keys_np, bits, ordering_len=None, with_visible=True):
    n = keys_np.size
    keys = torch.from_numpy(keys_np.view(np.int32)).cuda()
    ordering = torch.full((ordering_len or rb.align_capacity(n),), -1, dtype=torch.int32, device="cuda")
    visible = torch.zeros(1, dtype=torch.int32, device="cuda")
    vis_ptr = ctypes.c_void_p(visible.data_ptr()) if with_visible else None
    torch.cuda.synchronize()
    st = _abi.lib().rdx_sort_noalloc(ctypes.c_void_p(keys.data_ptr()), n, bits, ctypes.c_void_p(ordering.data_ptr()),
                                     ordering.numel(), vis_ptr, None)
    torch.cuda.synchronize()
    vis = int(visible.cpu().numpy().view(np.uint32)[0]) if with_visible else None
    return st, ordering.cpu().numpy().view(np.uint32), vis


# (keys, bits, seed, every k-th key invalid): 4096-key digit passes, 1024-key
# passes of small sorts (at most 256 tiles; their lookback words lie elsewhere
# in the array), 16-bit keys, and a tiny sort, one after another
CASES = [(300_000, 32, 1, 7), (MAX_KEYS, 24, 2, 3), (200_000, 16, 3, 5), (5_000, 32, 4, 2), (300_000, 32, 5, 0)]


def test_calls_in_a_row_match_rdx_sort_and_the_oracle():
    for n, bits, seed, every in CASES:
        keys = _keys(n, bits, seed, every)
        st, got, visible = _noalloc(keys, bits)
        assert st == _abi.RDX_OK, (n, bits)
        expected, exp_visible = rb.SortKeys.sort(torch.from_numpy(keys.view(np.int32)).cuda(), n, bits)
        torch.cuda.synchronize()
        assert visible == exp_visible, (n, bits)
        np.testing.assert_array_equal(got[:n], expected.cpu().numpy().view(np.uint32)[:n])
        assert (got[n:] == 0xFFFFFFFF).all()  # entries past count are left as they were
        order, orc_visible = orc.sort(keys, n, bits)
        assert visible == orc_visible, (n, bits)
        np.testing.assert_array_equal(got[:n], order[:n])


def test_without_visible_the_order_still_matches():
    keys = _keys(120_000, 24, 6, 4)
    st, got, _ = _noalloc(keys, 24, with_visible=False)
    assert st == _abi.RDX_OK
    expected, _ = rb.SortKeys.sort(torch.from_numpy(keys.view(np.int32)).cuda(), keys.size, 24)
    np.testing.assert_array_equal(got[:keys.size], expected.cpu().numpy().view(np.uint32)[:keys.size])


def test_rejects_sizes_beyond_the_scratch_and_host_memory():
    st, _, _ = _noalloc(np.zeros(MAX_KEYS + 1, dtype=np.uint32), 32)
    assert st == _abi.RDX_ERR_CAPACITY
    host = np.zeros(16, dtype=np.uint32)
    out = np.zeros(16, dtype=np.uint32)
    st = _abi.lib().rdx_sort_noalloc(host.ctypes.data, 16, 32, out.ctypes.data, 16, None, None)
    assert st == _abi.RDX_ERR_ARG
