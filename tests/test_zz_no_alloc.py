"""The scan entry point that allocates nothing (vox_global_scan_u64_noalloc).

It exists for callers that cannot let the library allocate device memory:
hosts whose device memory belongs to their own allocator (a framework's
caching pool that holds the free memory), and loops that cannot afford the
device synchronisation of cudaMalloc / cudaFree.  Its scratch is a fixed array
inside the library that every call shares and that keeps the last call's
contents, so this test calls it through the C ABI several times in a row and
compares each result exactly (integer scan) with the allocating entry point,
vox_global_scan_u64, and with numpy: sums past 2^55 and wrapping mod 2^64, an
empty input, both scan kinds.  It runs last so a failure here never hides
another test, and it works alone in a fresh process as well as after the rest
of the suite.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(lib):
    lib.vox_global_scan_u64_noalloc.restype = ctypes.c_int
    lib.vox_global_scan_u64_noalloc.argtypes = [
        ctypes.c_void_p,
        ctypes.c_void_p,
        ctypes.c_int64,
        ctypes.c_int,
        ctypes.c_void_p,
        ctypes.c_void_p,
    ]
    return lib.vox_global_scan_u64_noalloc


def _numpy_scan(x, inclusive):
    ref = np.cumsum(x, dtype=np.uint64)  # uint64 addition wraps mod 2^64
    if not inclusive and x.size:
        ref = np.concatenate([[np.uint64(0)], ref[:-1]]).astype(np.uint64)
    return ref


def test_noalloc_scan_matches_allocating_scan(vox_ctx):
    import torch

    noalloc = _bind(vox_ctx.lib)
    stream = torch.cuda.current_stream().cuda_stream
    # calls in a row on the shared scratch: each must see none of the previous one's words
    cases = (
        (3_000_001, 1, 1, 1 << 30),
        (123_457, 0, 2, 1 << 30),
        (1 << 24, 1, 3, 1 << 40),  # the size limit; the running sum passes 2^55
        (500_003, 0, 4, 1 << 62),  # wraps mod 2^64
        (0, 1, 5, 1),
    )
    for n, inclusive, seed, top in cases:
        x = np.random.default_rng(seed).integers(0, top, n, dtype=np.uint64)
        d_in = torch.from_numpy(x.view(np.int64)).cuda() if n else torch.zeros(1, dtype=torch.int64, device="cuda")
        d_ref = torch.empty_like(d_in)
        d_got = torch.full_like(d_in, -1)
        t_ref = torch.zeros(1, dtype=torch.int64, device="cuda")
        t_got = torch.full((1,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        if n:
            vox_ctx.global_scan_u64(d_in, d_ref, t_ref, bool(inclusive))
        rc = noalloc(d_in.data_ptr(), d_got.data_ptr(), n, inclusive, t_got.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        total = int(x.sum(dtype=np.uint64))
        assert int(t_got.cpu().numpy().view(np.uint64)[0]) == total
        if n:
            assert torch.equal(d_got, d_ref)
            assert int(t_ref.cpu().numpy().view(np.uint64)[0]) == total
            np.testing.assert_array_equal(d_got.cpu().numpy().view(np.uint64), _numpy_scan(x, inclusive))
        else:
            assert int(d_got.item()) == -1  # nothing written for an empty input


def test_noalloc_scan_rejects_oversize(vox_ctx):
    import torch

    noalloc = _bind(vox_ctx.lib)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    # the size check comes before any device work, so the pointers are never read
    dummy = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 24) + 1, 1, tot.data_ptr(), None)
    assert rc == -7  # VOX_ERR_SIZE
