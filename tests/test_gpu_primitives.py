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
