"""GPU tests of the parallel primitives exposed through the C ABI
(vox_global_scan_u64, vox_radix_sort_key64), checked the way the reference
checks its sort (raster/ParallelPrimitives.cpp:910-968: monotone keys and an
unchanged key checksum) plus exact comparison with numpy."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 1_000_003])
@pytest.mark.parametrize("inclusive", [True, False])
def test_scan_matches_numpy(vox_ctx, n, inclusive):
    import torch

    rng = np.random.default_rng(n + inclusive)
    x = rng.integers(0, 1 << 20, n, dtype=np.uint64)
    d_in = torch.from_numpy(x.view(np.int64)).cuda()
    d_out = torch.empty_like(d_in)
    d_tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    vox_ctx.global_scan_u64(d_in, d_out, d_tot, inclusive)
    got = d_out.cpu().numpy().view(np.uint64)
    ref = np.cumsum(x, dtype=np.uint64)
    if not inclusive:
        ref = np.concatenate([[0], ref[:-1]]).astype(np.uint64) if n else ref
    np.testing.assert_array_equal(got, ref)
    assert int(d_tot.cpu().numpy().view(np.uint64)[0]) == int(x.sum())


def _scan_ref(x, inclusive):
    ref = np.cumsum(x, dtype=np.uint64)  # numpy uint64 addition wraps mod 2^64
    if not inclusive and x.size:
        ref = np.concatenate([[np.uint64(0)], ref[:-1]]).astype(np.uint64)
    return ref


@pytest.mark.parametrize("n", [2049, 700_001])
@pytest.mark.parametrize("top", [1 << 40, 1 << 50, 1 << 62])
def test_scan_full_64_bit_prefixes(vox_ctx, n, top):
    # running sums that pass 2^55 (top 2^40 and 2^50 over many tiles) and wrap
    # mod 2^64 (top 2^62): the reference's global_scan_uint64
    # (raster/ParallelPrimitives.cpp:151-310) is plain uint64 arithmetic
    import torch

    rng = np.random.default_rng(n ^ top)
    x = rng.integers(0, top, n, dtype=np.uint64)
    for inclusive in (True, False):
        d_in = torch.from_numpy(x.view(np.int64)).cuda()
        d_out = torch.empty_like(d_in)
        d_tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        vox_ctx.global_scan_u64(d_in, d_out, d_tot, inclusive)
        np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint64), _scan_ref(x, inclusive))
        assert int(d_tot.cpu().numpy().view(np.uint64)[0]) == int(x.sum(dtype=np.uint64))
    if top == 1 << 40 and n > 100_000:
        assert int(np.cumsum(x, dtype=np.uint64)[-1]) > (1 << 55)


@pytest.mark.parametrize("n,bits", [(2, 64), (8191, 17), (8193, 64), (12_993_895, 64), (3_000_000, 33)])
def test_radix_sort_key64(vox_ctx, n, bits):
    # 12,993,895 random 64-bit keys: the size of the reference's self-test
    import torch

    rng = np.random.default_rng(n)
    keys = rng.integers(0, np.iinfo(np.uint64).max, n, dtype=np.uint64, endpoint=True)
    if bits < 64:
        keys &= np.uint64((1 << bits) - 1)
    vals = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    torch.cuda.synchronize()
    vox_ctx.radix_sort_key64(dk, dv, bits)
    gk = dk.cpu().numpy().view(np.uint64)
    gv = dv.cpu().numpy().view(np.uint32)
    assert np.all(gk[1:] >= gk[:-1])
    assert int(np.bitwise_xor.reduce(gk)) == int(np.bitwise_xor.reduce(keys))
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(gk, keys[order])
    np.testing.assert_array_equal(gv, vals[order])


def test_sort_partial_key_bits_is_stable(vox_ctx):
    import torch

    n = 100_000
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 1 << 40, n, dtype=np.uint64)
    vals = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    torch.cuda.synchronize()
    vox_ctx.radix_sort_key64(dk, dv, 8)  # only the low byte
    gk = dk.cpu().numpy().view(np.uint64)
    order = np.argsort(keys & np.uint64(255), kind="stable")
    np.testing.assert_array_equal(gk, keys[order])


def _dev(a, dtype):
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a).view(dtype).copy()).cuda()
    torch.cuda.synchronize()
    return t


@pytest.mark.parametrize("n", [0, 1, 2047, 2049, 700_001])
@pytest.mark.parametrize("inclusive", [True, False])
def test_scan_u32_wraps_like_reference(vox_ctx, n, inclusive):
    # the reference's global_scan: uint32 sums that wrap mod 2^32
    import torch

    rng = np.random.default_rng(n + 7 * inclusive)
    x = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    d_in, d_out = _dev(x, np.int32), torch.empty(n, dtype=torch.int32, device="cuda")
    d_tot = torch.zeros(1, dtype=torch.int32, device="cuda")
    vox_ctx.global_scan_u32(d_in, d_out, d_tot, inclusive)
    ref = np.cumsum(x.astype(np.uint64)) & np.uint64(0xFFFFFFFF)
    if not inclusive and n:
        ref = np.concatenate([[0], ref[:-1]])
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), ref.astype(np.uint32))
    assert int(d_tot.cpu().numpy().view(np.uint32)[0]) == int(x.astype(np.uint64).sum()) % (1 << 32)


@pytest.mark.parametrize("n", [1, 2048, 2049, 1_000_003])
def test_scan_max_u32(vox_ctx, n):
    # the reference's global_scan_max: inclusive running maximum
    import torch

    rng = np.random.default_rng(n)
    x = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    x[::3] = rng.integers(0, 1000, len(x[::3])).astype(np.uint32)
    d_in, d_out = _dev(x, np.int32), torch.empty(n, dtype=torch.int32, device="cuda")
    vox_ctx.global_scan_max_u32(d_in, d_out)
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint32), np.maximum.accumulate(x))


@pytest.mark.parametrize("n,bits", [(2, 32), (9_000, 20), (3_000_001, 32), (500_000, 13)])
def test_radix_sort_u32_partial_bits(vox_ctx, n, bits):
    # only key bits [0, bits) order the pairs; the others ride along
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = _dev(keys, np.int32), _dev(vals, np.int32)
    vox_ctx.radix_sort_u32(dk, dv, bits)
    order = np.argsort(keys & np.uint32((1 << bits) - 1 if bits < 32 else 0xFFFFFFFF), kind="stable")
    np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint32), keys[order])
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("n,bits", [(100_000, 20), (70_000, 41)])
def test_radix_sort_key64_ignores_bits_above_count(vox_ctx, n, bits):
    rng = np.random.default_rng(bits)
    keys = rng.integers(0, np.iinfo(np.uint64).max, n, dtype=np.uint64, endpoint=True)
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = _dev(keys, np.int64), _dev(vals, np.int32)
    vox_ctx.radix_sort_key64(dk, dv, bits)
    order = np.argsort(keys & np.uint64((1 << bits) - 1), kind="stable")
    np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("n,low_bits,high_bits", [(2, 32, 1), (50_000, 32, 10), (400_001, 16, 7), (9_999, 32, 0)])
def test_radix_sort_dual_key(vox_ctx, n, low_bits, high_bits):
    # the tile sort of raster_gaussian_2d: (tile id, depth) with the tile id in
    # the high key (raster/Raster2D.cpp:495-506)
    rng = np.random.default_rng(n + low_bits)
    low = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    high = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    vals = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    dl, dh, dv = _dev(low, np.int32), _dev(high, np.int32), _dev(vals, np.int32)
    vox_ctx.radix_sort_dual_key(dl, dh, dv, low_bits, high_bits)
    ml = np.uint32((1 << low_bits) - 1 if low_bits < 32 else 0xFFFFFFFF)
    mh = np.uint32((1 << high_bits) - 1 if high_bits < 32 else 0xFFFFFFFF)
    order = np.lexsort((np.arange(n), low & ml, high & mh))  # last key primary; index keeps it stable
    np.testing.assert_array_equal(dl.cpu().numpy().view(np.uint32), low[order])
    np.testing.assert_array_equal(dh.cpu().numpy().view(np.uint32), high[order])
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("cand", list(range(10)))
def test_every_sort_candidate_is_the_same_stable_sort(cand):
    # VOX_SORT_SHAPE fixes the tuner's candidate: 0-4 onesweep tile shapes
    # (decoupled look-back), 5-9 the same tiles as three-kernel passes (tile
    # digit counts, per-digit offsets, scatter); all are the same stable sort
    import os

    import torch

    from nanovdb_editor.vox import VoxContext

    os.environ["VOX_SORT_SHAPE"] = str(cand)
    try:
        ctx = VoxContext(0)
    finally:
        del os.environ["VOX_SORT_SHAPE"]
    try:
        for n, bits in ((1, 32), (4097, 20), (300_001, 31), (2_000_003, 64)):
            rng = np.random.default_rng(1000 * cand + n)
            if bits == 64:
                keys = rng.integers(0, np.iinfo(np.uint64).max, n, dtype=np.uint64, endpoint=True)
                vals = np.arange(n, dtype=np.uint32)
                dk, dv = _dev(keys, np.int64), _dev(vals, np.int32)
                ctx.radix_sort_key64(dk, dv, bits)
                gk = dk.cpu().numpy().view(np.uint64)
            else:
                keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
                keys[: n // 3] = keys[0]  # long runs of equal keys: stability
                vals = np.arange(n, dtype=np.uint32)
                dk, dv = _dev(keys, np.int32), _dev(vals, np.int32)
                ctx.radix_sort_u32(dk, dv, bits)
                gk = dk.cpu().numpy().view(np.uint32)
            torch.cuda.synchronize()
            order = np.argsort(keys, kind="stable")
            np.testing.assert_array_equal(gk, keys[order])
            np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])
    finally:
        ctx.close()
