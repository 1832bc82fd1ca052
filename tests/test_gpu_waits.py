"""The bounded device waits (decoupled look-back of the scans and the onesweep
sort) running out: with vox_context_set_wait_limit withholding every tile's
publication, each wait polls a word nothing writes until its limit, the
kernels finish, and the call returns VOX_ERR_TIMEOUT; the same context then
succeeds on normal calls.  No fault, trap or endless wait: only the bound of a
wait that already returns is shortened."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_scan_and_sort_time_out_then_recover(vox_ctx):
    import torch
    from nanovdb_editor.exceptions import PipelineError
    from nanovdb_editor.vox import VoxContext

    ctx = VoxContext(0)
    try:
        n = 200_003
        rng = np.random.default_rng(7)
        x = rng.integers(0, 1 << 40, n, dtype=np.uint64)
        keys = rng.integers(0, 1 << 62, n, dtype=np.uint64)
        vals = np.arange(n, dtype=np.uint32)

        def run_scan():
            d_in = torch.from_numpy(x.view(np.int64)).cuda()
            d_out = torch.empty_like(d_in)
            d_tot = torch.zeros(1, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            ctx.global_scan_u64(d_in, d_out, d_tot, True)
            return d_out.cpu().numpy().view(np.uint64)

        def run_sort():
            dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
            dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
            torch.cuda.synchronize()
            ctx.radix_sort_key64(dk, dv, 64)
            return dk.cpu().numpy().view(np.uint64), dv.cpu().numpy().view(np.uint32)

        ctx.set_wait_limit(1000, withhold_publication=True)
        with pytest.raises(PipelineError, match="bounded device wait expired"):
            run_scan()
        with pytest.raises(PipelineError, match="bounded device wait expired"):
            run_sort()
        ctx.set_wait_limit(None)
        np.testing.assert_array_equal(run_scan(), np.cumsum(x, dtype=np.uint64))
        gk, gv = run_sort()
        order = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(gk, keys[order])
        np.testing.assert_array_equal(gv, vals[order])
        # a limit alone (publication on) leaves results exact
        ctx.set_wait_limit(1 << 20)
        np.testing.assert_array_equal(run_scan(), np.cumsum(x, dtype=np.uint64))
    finally:
        ctx.close()
