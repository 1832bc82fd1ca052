"""The scan entry point that allocates nothing (vox_global_scan_u64_noalloc).

It exists for callers that cannot let the library allocate device memory:
hosts whose device memory belongs to their own allocator, and loops that
cannot afford the device synchronisation of cudaMalloc / cudaFree.  Its
scratch is a fixed array inside the library, so this test calls it through
the C ABI twice in a row and compares each result with the allocating entry
point, vox_global_scan_u64, exactly (integer scan).  It runs last so a
failure here never hides another test, and it works alone in a fresh process
as well as after the rest of the suite.
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


def test_noalloc_scan_matches_allocating_scan(vox_ctx):
    import torch

    noalloc = _bind(vox_ctx.lib)
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row: the second must not see the first one's scratch
    for n, inclusive, seed in ((3_000_001, 1, 1), (123_457, 0, 2)):
        x = np.random.default_rng(seed).integers(0, 1 << 30, n, dtype=np.uint64)
        d_in = torch.from_numpy(x.view(np.int64)).cuda()
        d_ref = torch.empty_like(d_in)
        d_got = torch.full_like(d_in, -1)
        t_ref = torch.zeros(1, dtype=torch.int64, device="cuda")
        t_got = torch.full((1,), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        vox_ctx.global_scan_u64(d_in, d_ref, t_ref, bool(inclusive))
        rc = noalloc(d_in.data_ptr(), d_got.data_ptr(), n, inclusive, t_got.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert torch.equal(d_got, d_ref)
        assert int(t_got.item()) == int(t_ref.item()) == int(x.sum())


def test_noalloc_scan_rejects_oversize(vox_ctx):
    import torch

    noalloc = _bind(vox_ctx.lib)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    # the size check comes before any device work, so the pointers are never read
    dummy = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 24) + 1, 1, tot.data_ptr(), None)
    assert rc == -7  # VOX_ERR_SIZE
