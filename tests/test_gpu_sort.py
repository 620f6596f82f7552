"""The CUDA sorts against SortKeys.sort (the oracle): the reference's grid of
widths and counts (test/gpu/renderTests.ts:31-57), compaction then an
indirect sort (renderTests.ts:59-90), the splat sorter (renderTests.ts:369-390),
keys from distances, host and device buffers, and ties."""
import numpy as np
import pytest
import torch

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200 import _abi
from radix_b200.synthetic import Mulberry32
from tests.parity import host, to_cuda, u32

pytestmark = pytest.mark.gpu
BITS = (16, 24, 32)


def random_keys(n, bits, seed):
    return (Mulberry32(seed).uniform(max(n, 1)) * 2.0 ** bits).astype(np.uint64).astype(np.uint32)


@pytest.mark.parametrize("bits", BITS)
@pytest.mark.parametrize("count", [0, 1, 4095, 4096, 4097, 70000, 1_000_003])
def test_radix_sort_pairs_equals_sort_keys(ctx, bits, count):
    keys = random_keys(count, bits, 7 + count + bits)
    vals = np.arange(max(count, 1), dtype=np.uint32)
    kt, vt = to_cuda(keys.view(np.int32)), to_cuda(vals.view(np.int32))
    rb.RadixSort(kt, vt, ctx).sort(count, bits)
    expected, _ = orc.sort(keys, count, bits)
    got = u32(vt)[:count]
    np.testing.assert_array_equal(got, expected[:count])
    np.testing.assert_array_equal(u32(kt)[:count], keys[expected[:count]])


@pytest.mark.parametrize("bits", BITS)
def test_sort_keys_sort_ordering_visible_and_untouched_tail(ctx, bits):
    n = 300_000
    keys = random_keys(n, bits, 3)
    keys[::7] = rb.SortKeys.invalid(bits)
    ordering = torch.full((rb.align_capacity(n),), 12345, dtype=torch.int32, device="cuda")
    got, visible = rb.SortKeys.sort(to_cuda(keys.view(np.int32)), n, bits, ordering=ordering, ctx=ctx)
    expected, exp_visible = orc.sort(keys, n, bits)
    assert visible == exp_visible
    np.testing.assert_array_equal(u32(got)[:n], expected[:n])
    assert (host(got)[n:] == 12345).all()


def test_sort_from_and_to_host_memory(ctx):
    n = 50_000
    keys = random_keys(n, 24, 5)
    ordering = np.zeros(rb.align_capacity(n), dtype=np.uint32)
    got, visible = rb.SortKeys.sort(keys, n, 24, ordering=ordering, ctx=ctx)
    expected, exp_visible = orc.sort(keys, n, 24)
    assert got is ordering and visible == exp_visible
    np.testing.assert_array_equal(ordering, expected)


def test_sort_short_ordering_raises_the_reference_message(ctx):
    with pytest.raises(rb.RadixError, match="SortKeys.sort: ordering holds 10 of 20 indices"):
        rb.SortKeys.sort(np.zeros(20, dtype=np.uint32), 20, 32, ordering=np.zeros(10, dtype=np.uint32), ctx=ctx)
    with pytest.raises(rb.RadixError, match="bits must be 16, 24 or 32"):
        rb.SortKeys.sort(np.zeros(20, dtype=np.uint32), 20, 20, ctx=ctx)


@pytest.mark.parametrize("pattern", ["equal", "three", "descending", "ascending", "upper_bits"])
def test_sort_ties_and_patterns(ctx, pattern):
    n = 200_000
    if pattern == "equal":
        keys = np.full(n, 0x1234, dtype=np.uint32)
    elif pattern == "three":
        keys = (random_keys(n, 32, 9) % 3).astype(np.uint32) * 0x01010101
    elif pattern == "descending":
        keys = np.arange(n, 0, -1, dtype=np.uint32)
    elif pattern == "ascending":
        keys = np.arange(n, dtype=np.uint32)
    else:  # bits above the width: the 16-bit layout ignores them
        keys = random_keys(n, 32, 11)
    bits = 16 if pattern == "upper_bits" else 32
    got, visible = rb.SortKeys.sort(to_cuda(keys.view(np.int32)), n, bits, ctx=ctx)
    expected, exp_visible = orc.sort(keys, n, bits)
    assert visible == exp_visible
    np.testing.assert_array_equal(u32(got)[:n], expected[:n])


@pytest.mark.parametrize("bits", BITS)
def test_compact_then_sort_indirect_equals_sort_keys(ctx, bits):
    n = 20000
    rng = Mulberry32(11)
    u = rng.uniform(n)
    v = rng.uniform(n)
    keys = np.where(u < 0.3, rb.SortKeys.invalid(bits), (v * 0xFF * 2 ** (bits - 8)).astype(np.uint64)).astype(np.uint32)
    ck, cv, count = rb.Compact(ctx, invalid=rb.SortKeys.invalid(bits)).compact(to_cuda(keys.view(np.int32)))
    rb.RadixSort(ck, cv, ctx).sort_indirect(count, bits)
    ordering, visible = orc.sort(keys, n, bits)
    assert int(u32(count)[0]) == visible
    np.testing.assert_array_equal(u32(cv)[:visible], ordering[:visible])


def test_compact_keeps_input_order(ctx):
    n = 1_000_000
    keys = random_keys(n, 32, 4)
    keys[Mulberry32(2).uniform(n) < 0.5] = 0xFFFFFFFF
    ck, cv, count = rb.Compact(ctx).compact(to_cuda(keys.view(np.int32)))
    idx = np.flatnonzero(keys != 0xFFFFFFFF)
    assert int(u32(count)[0]) == idx.size
    np.testing.assert_array_equal(u32(cv)[:idx.size], idx)
    np.testing.assert_array_equal(u32(ck)[:idx.size], keys[idx])


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 70_001, 4096 * 1030 + 7])
@pytest.mark.parametrize("valid", [0.0, 0.5, 1.0])
def test_compact_ragged_sizes_and_fractions(ctx, n, valid):
    """Tile edges (4096 keys a tile, more tiles than the scan's 1024 threads),
    no valid key, every key valid, and an invalid value other than the largest
    key: the kept keys and their indices in input order, and their count."""
    invalid = 0x00ABCDEF
    keys = random_keys(n, 32, n + 3) if n else np.zeros(0, np.uint32)
    keys[keys == invalid] = 0
    keys[Mulberry32(7).uniform(n) >= valid] = invalid
    ck, cv, count = rb.Compact(ctx, invalid=invalid).compact(to_cuda(keys.view(np.int32)) if n else
                                                          torch.zeros(1, dtype=torch.int32, device="cuda"), n)
    idx = np.flatnonzero(keys != invalid)
    assert int(u32(count)[0]) == idx.size
    np.testing.assert_array_equal(u32(cv)[:idx.size], idx)
    np.testing.assert_array_equal(u32(ck)[:idx.size], keys[idx])


def test_compact_from_host_buffers(ctx):
    """The same call with host (numpy) buffers: copies in and out around the launches."""
    n = 300_001
    keys = random_keys(n, 32, 5)
    keys[::4] = 0xFFFFFFFF
    ck, cv, count = rb.Compact(ctx).compact(keys)
    idx = np.flatnonzero(keys != 0xFFFFFFFF)
    assert int(count[0]) == idx.size
    np.testing.assert_array_equal(cv[:idx.size].view(np.uint32), idx)
    np.testing.assert_array_equal(ck[:idx.size].view(np.uint32), keys[idx])


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("bits", [24, 32])
def test_keys_sharing_one_top_digit(ctx, bits, variant):
    """Every valid key has the same top byte (depths within one top-byte range):
    the cooperative passes skip the top pass, which would keep the order; every
    variant's order equals the oracle's."""
    n = 300_001
    rng = Mulberry32(17 + bits)
    low = (rng.uniform(n) * 2.0 ** (bits - 8)).astype(np.uint64).astype(np.uint32)
    low[::7] = low[3]  # ties
    keys = (np.uint32(0xA5) << np.uint32(bits - 8)) | low
    keys[Mulberry32(19).uniform(n) < 0.3] = rb.SortKeys.invalid(bits)
    ctx.set_sort_variant(variant)
    try:
        got, visible = rb.SortKeys.sort(to_cuda(keys.view(np.int32)), n, bits, ctx=ctx)
        kt, vt = to_cuda(keys.view(np.int32)), torch.arange(n, dtype=torch.int32, device="cuda")
        rb.RadixSort(kt, vt, ctx).sort(n, bits)
    finally:
        ctx.set_sort_variant(-1)
    expected, exp_visible = orc.sort(keys, n, bits)
    assert visible == exp_visible
    np.testing.assert_array_equal(u32(got)[:n], expected[:n])
    np.testing.assert_array_equal(u32(vt), expected[:n])


@pytest.mark.parametrize("bits", BITS)
def test_splat_sorter_values_count_and_draw_args(ctx, bits):
    n = 123_457
    keys = random_keys(n, bits - 1, 13)
    keys[Mulberry32(5).uniform(n) < 0.25] = rb.SortKeys.invalid(bits)
    sorter = rb.SplatSorter(ctx)
    values, count, args = sorter.sort(to_cuda(keys.view(np.int32)), n, bits)
    ordering, visible = orc.sort(keys, n, bits)
    assert sorter.read_count() == visible
    q = rb.SplatSorter.QUADS_PER_INSTANCE
    assert list(u32(args)) == [6 * q, -(-visible // q), 0, 0, 0]
    np.testing.assert_array_equal(u32(values)[:visible], ordering[:visible])


@pytest.mark.parametrize("bits", BITS)
def test_keys_compute_bit_exact(ctx, bits):
    rng = Mulberry32(21)
    d = np.concatenate([
        np.exp(rng.uniform(100_000) * 80 - 40),
        [0.0, -0.0, 1e-45, 1e-40, 1.0, 2.0 ** -32, 2.0 ** 32, 3e38, 4e38, 1e300, np.inf, -np.inf, np.nan, -1.0],
    ])
    got = u32(rb.SortKeys.compute(to_cuda(d), bits, ctx))
    np.testing.assert_array_equal(got, orc.sort_keys(d, bits))
    d32 = d.astype(np.float32)
    ref32 = np.array([orc.sort_key_f32(x, bits) for x in d32], dtype=np.uint32)
    got32 = u32(rb.SortKeys.compute(to_cuda(d32), bits, ctx))
    np.testing.assert_array_equal(got32, ref32)
    # distances not 16-byte aligned (the scalar kernels) and lengths of every remainder mod 4
    for off in (1, 2, 3):
        for cut in (0, 1, 2, 3):
            end = d.size - cut
            got = u32(rb.SortKeys.compute(to_cuda(d)[off:end], bits, ctx))
            np.testing.assert_array_equal(got, orc.sort_keys(d[off:end], bits), err_msg=f"f64 {off} {cut}")
            got32 = u32(rb.SortKeys.compute(to_cuda(d32)[off:end], bits, ctx))
            np.testing.assert_array_equal(got32, ref32[off:end], err_msg=f"f32 {off} {cut}")


def test_sort_large_random_32bit(ctx):
    n = 4_000_000
    keys = random_keys(n, 32, 99)
    got, visible = rb.SortKeys.sort(to_cuda(keys.view(np.int32)), n, 32, ctx=ctx)
    expected, exp_visible = orc.sort(keys, n, 32)
    assert visible == exp_visible
    np.testing.assert_array_equal(u32(got)[:n], expected[:n])


@pytest.mark.parametrize("n", [256 * 4096, 256 * 4096 + 1])
def test_sort_keys_sort_at_the_small_tile_threshold(ctx, n):
    """Up to 256 tiles of 4096 keys the digit passes run in 1024-key tiles; one
    key more and they do not: both orders equal the oracle's."""
    keys = random_keys(n, 32, 11)
    keys[::3] = rb.SortKeys.invalid(32)
    got, visible = rb.SortKeys.sort(to_cuda(keys.view(np.int32)), n, 32, ctx=ctx)
    expected, exp_visible = orc.sort(keys, n, 32)
    assert visible == exp_visible
    np.testing.assert_array_equal(u32(got)[:n], expected[:n])


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("bits", [24, 32])
def test_a_wait_that_runs_out_reports_a_timeout_and_the_context_recovers(bits, variant):
    """A test hook silences one digit pass: with onesweep passes (variant 0)
    its first tile publishes no lookback word, in the cooperative kernel
    (variant 1) block 0 does not arrive at the pass's grid barrier. The waits
    on it run out after 64 polls: the call returns RDX_ERR_TIMEOUT with its
    text, every kernel finishes, and the same context then sorts bit-exact
    again (the reference throws on misuse, src/wgpu/WgpuRadixSort.ts:150-152;
    it has no device waits)."""
    c = rb.Context(0)
    c.set_sort_variant(variant)
    n = 150_000
    keys = random_keys(n, bits, 21)
    keys[::3] = rb.SortKeys.invalid(bits)
    expected, visible = orc.sort(keys, n, bits)
    for silent_pass in range(bits // 8):
        c.set_wait(64, silent_pass)
        with pytest.raises(rb.RadixError) as e:
            rb.SortKeys.sort(keys, n, bits, ctx=c)  # host buffers: the call synchronises
        assert e.value.code == _abi.RDX_ERR_TIMEOUT
        assert "device wait gave up" in str(e.value)
        c.set_wait(0, -1)
        order, vis = rb.SortKeys.sort(keys, n, bits, ctx=c)
        assert vis == visible
        np.testing.assert_array_equal(u32(order)[:n], expected[:n])
    c.close()


SIZES = [0, 1, 4095, 4096, 4097, 70000, 1_000_003, 4_000_000]


@pytest.mark.parametrize("variant", range(7))
@pytest.mark.parametrize("bits", BITS)
def test_every_digit_pass_variant_sorts_bit_exact(variant, bits):
    """Onesweep passes with tiles by size (0) or of 4096, 2048 and 1024 keys
    (4-6) and the cooperative kernel's variants (1-3: 1024x16, 512x16, 1024x8
    threads x keys): SortKeys.sort (partition, then the valid keys) and
    WgpuRadixSort.sort (in place, every key ranked) on the reference grid, up
    to 4M keys (several sub-tiles a block)."""
    c = rb.Context(0)
    c.set_sort_variant(variant)
    for count in SIZES:
        keys = random_keys(count, bits, 100 + count + bits + variant)
        if count:
            keys[::5] = rb.SortKeys.invalid(bits)
        expected, visible = orc.sort(keys, count, bits)
        order, vis = rb.SortKeys.sort(to_cuda(keys.view(np.int32)), count, bits, ctx=c)
        torch.cuda.synchronize()
        assert vis == visible, (variant, bits, count)
        np.testing.assert_array_equal(u32(order)[:count], expected[:count], err_msg=f"{variant} {bits} {count}")
        kt, vt = to_cuda(keys.view(np.int32)), to_cuda(np.arange(max(count, 1), dtype=np.int32))
        rb.RadixSort(kt, vt, c).sort(count, bits)
        np.testing.assert_array_equal(u32(vt)[:count], expected[:count], err_msg=f"pairs {variant} {bits} {count}")
        np.testing.assert_array_equal(u32(kt)[:count], keys[expected[:count]])
    c.close()


@pytest.mark.parametrize("variant", range(7))
def test_every_digit_pass_variant_gives_the_frame_order(variant):
    from radix_b200 import synthetic as syn
    d = syn.mixture_table(1_000_000, seed=4, sh_degree=1)
    cam = syn.scale_camera()
    c = rb.Context(0)
    c.set_sort_variant(variant)
    t = rb.Table.from_dict(d, to=to_cuda)
    res = rb.frame([rb.SplatObject(t)], cam, None, 32, ("keys",), ctx=c)
    keys = u32(res["keys"])
    expected, visible = orc.sort(keys, keys.size, 32)
    assert res["visible"] == visible
    np.testing.assert_array_equal(u32(res["ordering"]), expected[:keys.size])
    batch = rb.Batch([([rb.SplatObject(t)], cam)], None, 32, ("keys",), ctx=c)
    for _ in range(2):
        batch.launch()
        batch.synchronize()
        np.testing.assert_array_equal(u32(batch.results()["ordering"]), expected[:keys.size])
    batch.close()
    c.close()
