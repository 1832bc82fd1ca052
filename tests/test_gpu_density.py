"""Parity at the benchmark's density and on the benchmark's own batch.

1. Four planar clusters of 31,250 Gaussians at voxel 0.002: the per-cluster
   density of the 2M / 64-cluster workload the bench times (about 1.0e8
   passing (voxel, Gaussian) pairs, 5.3e8 tested voxels, 63 of the
   reference's 8M-fragment windows).  The CUDA path in the reference's node
   order against the oracle's window-by-window build: every node2 byte, the
   sorted pair list (by count and SHA-256), RGBA8 and the float channels bit
   for bit, and the float density's error against the oracle's FP64 sums,
   stated and bounded by 1e-5 of the grid's maximum.
2. The bench's 256-cloud uneven batch (9.0M Gaussians): every cloud's grid
   from the one batched call is byte-identical to its single-cloud grid, and
   the two smallest clouds match the oracle.
"""

import hashlib

import numpy as np
import pytest

from nanovdb_editor import workloads as W

pytestmark = pytest.mark.gpu

NAMES = ("means", "quats", "scales", "opacities", "colors")


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_headline_density_matches_oracle(vox_ctx, oracle_mod):
    from nanovdb_editor.vox import FLAG_WINDOW_ORDER

    cloud = W.cluster_cloud(125_000, 1, clusters=4)
    vs = 0.002
    g = vox_ctx.voxelize_host(*[cloud[k] for k in NAMES], vs, 0.05, FLAG_WINDOW_ORDER)
    ref = oracle_mod.OracleResult(cloud, vs, 0.05, window_mode=1)
    try:
        assert ref.counts["windows"] > 1
        assert g.counts["pairs"] == ref.counts["P"] and g.counts["voxels"] == ref.counts["V"], (g.counts, ref.counts)
        assert np.array_equal(g.node2, ref.node2()), "node2 region differs from the oracle's window build"
        vals = ref.values()
        np.testing.assert_array_equal(g.rgba8, vals["rgba8"])
        np.testing.assert_array_equal(g.density, vals["density"])
        np.testing.assert_array_equal(g.color, vals["color"])
        dmax = float(np.abs(vals["density64"]).max())
        err = float(np.abs(g.density.astype(np.float64) - vals["density64"]).max())
        print(f"headline density: P={ref.counts['P']} V={ref.counts['V']} windows={ref.counts['windows']} "
              f"max |f32 - f64| density = {err:.3g} (max {dmax:.3g}, {err / dmax:.2e} of max)")
        assert err <= 1e-5 * dmax
        k_ref, i_ref = ref.pairs()
        k, i = vox_ctx.pairs()
        assert k.size == k_ref.size
        assert _sha(k, i) == _sha(k_ref, i_ref), "sorted (voxel key, Gaussian) pairs differ from the oracle's"
    finally:
        ref.close()


def test_bench_batch_matches_single_calls(vox_ctx, oracle_mod):
    import torch

    import bench

    B = bench.BATCHED
    clouds, start, vs = W.batch_clouds(B["clouds"], 3, B["min_n"], B["max_n"])
    allc = W.concat(clouds)
    dev = [torch.from_numpy(np.ascontiguousarray(allc[k])).cuda() for k in NAMES]
    _, goff, voff = vox_ctx.voxelize_batch(*dev, start, vs)
    grids = vox_ctx.grids(goff)
    assert len(grids) == len(clouds) == B["clouds"] and int(start[-1]) > 8_000_000
    for b, (c, v) in enumerate(zip(clouds, vs)):
        single = vox_ctx.voxelize_host(*[c[k] for k in NAMES], float(v))
        assert np.array_equal(grids[b].buf, single.buf), f"cloud {b}: batched grid differs from its single-cloud grid"
        assert int(voff[b + 1] - voff[b]) == single.value_count
    _, goff, voff = vox_ctx.voxelize_batch(*dev, start, vs)  # the grids of the batched call again
    grids = vox_ctx.grids(goff)
    for b in np.argsort([c.n for c in clouds])[:2]:
        ref = oracle_mod.OracleResult(clouds[b], float(vs[b]), 0.05, window_mode=0)
        assert np.array_equal(grids[b].node2, ref.node2())
        vals = ref.values()
        np.testing.assert_array_equal(grids[b].rgba8, vals["rgba8"])
        np.testing.assert_array_equal(grids[b].density, vals["density"])
        ref.close()
