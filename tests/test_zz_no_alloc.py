"""rdx_sort_noalloc against rdx_sort, through the C ABI.

rdx_sort_noalloc serves callers that may not allocate GPU memory (hosts that
own the device memory budget, frame loops that cannot afford an allocation's
synchronisation): its scratch is a fixed array inside the library. Two calls in
a row must each give rdx_sort's order and visible count - the second one finds
the array as the first left it. This file is collected last so that a run
stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

import radix_b200 as rb
from radix_b200 import _abi
from radix_b200.synthetic import Mulberry32

pytestmark = pytest.mark.gpu
MAX_KEYS = 1 << 20


def _keys(n, bits, seed, invalid_every=0):
    k = (Mulberry32(seed).uniform(n) * 2.0 ** bits).astype(np.uint64).astype(np.uint32)
    if invalid_every:
        k[::invalid_every] = rb.SortKeys.invalid(bits)
    return k


def _noalloc(keys_np, bits, ordering_len=None):
    n = keys_np.size
    keys = torch.from_numpy(keys_np.view(np.int32)).cuda()
    ordering = torch.full((ordering_len or rb.align_capacity(n),), -1, dtype=torch.int32, device="cuda")
    visible = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = _abi.lib().rdx_sort_noalloc(ctypes.c_void_p(keys.data_ptr()), n, bits, ctypes.c_void_p(ordering.data_ptr()),
                                     ordering.numel(), ctypes.c_void_p(visible.data_ptr()), None)
    torch.cuda.synchronize()
    return st, ordering.cpu().numpy().view(np.uint32), int(visible.cpu().numpy().view(np.uint32)[0])


def test_two_calls_in_a_row_match_rdx_sort():
    cases = [(300_000, 32, 1, 7), (MAX_KEYS, 24, 2, 3)]
    for n, bits, seed, every in cases:
        keys = _keys(n, bits, seed, every)
        st, got, visible = _noalloc(keys, bits)
        assert st == _abi.RDX_OK
        expected, exp_visible = rb.SortKeys.sort(torch.from_numpy(keys.view(np.int32)).cuda(), n, bits)
        torch.cuda.synchronize()
        assert visible == exp_visible
        np.testing.assert_array_equal(got[:n], expected.cpu().numpy().view(np.uint32)[:n])
        assert (got[n:] == 0xFFFFFFFF).all()  # entries past count are left as they were


def test_rejects_sizes_beyond_the_scratch_and_host_memory():
    st, _, _ = _noalloc(np.zeros(MAX_KEYS + 1, dtype=np.uint32), 32)
    assert st == _abi.RDX_ERR_CAPACITY
    host = np.zeros(16, dtype=np.uint32)
    out = np.zeros(16, dtype=np.uint32)
    st = _abi.lib().rdx_sort_noalloc(host.ctypes.data, 16, 32, out.ctypes.data, 16, None, None)
    assert st == _abi.RDX_ERR_ARG
