"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bit-exact: sorted (voxel key, Gaussian id) pairs, the node2 region (masks,
prefix sums, child offsets, node counts, value indices, root keys), the
active-voxel bbox, RGBA8 values and the float32 density / colour sums (same
per-pair arithmetic, same sequential order).  Against the FP64 oracle the
float density and colour agree to 1e-5 of the grid's maximum density.
"""

import numpy as np
import pytest

from nanovdb_editor import workloads as W

pytestmark = pytest.mark.gpu

TOL_REL_MAX = 1e-5  # |f32 - f64| <= 1e-5 * max |density f64|


def _check(vox_ctx, oracle_mod, cloud, vs, cull=0.05):
    g = vox_ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"], vs, cull)
    ref = oracle_mod.OracleResult(cloud, vs, cull, window_mode=0)
    c = ref.counts
    assert c["error"] == 0
    got = g.counts
    assert got["pairs"] == c["P"]
    assert got["candidates"] == c["F"]
    assert got["voxels"] == c["V"]
    assert (got["upper"], got["lower"], got["leaf"]) == (c["upper"], c["lower"], c["leaf"])
    k_ref, i_ref = ref.pairs()
    k_got, i_got = vox_ctx.pairs()
    np.testing.assert_array_equal(k_got, k_ref)
    np.testing.assert_array_equal(i_got, i_ref)
    n2 = ref.node2()
    assert g.node2.shape == n2.shape
    if not np.array_equal(g.node2, n2):
        bad = np.nonzero(g.node2.view(np.uint64) != n2.view(np.uint64))[0]
        pytest.fail(f"node2 differs in {bad.size} words, first word index {bad[:8]}")
    if c["V"]:
        np.testing.assert_array_equal(g.bbox, ref.bbox())
    v = ref.values()
    np.testing.assert_array_equal(g.rgba8, v["rgba8"])
    np.testing.assert_array_equal(g.density, v["density"])
    np.testing.assert_array_equal(g.color, v["color"])
    dmax = float(np.abs(v["density64"]).max()) if c["V"] else 1.0
    err_d = float(np.abs(g.density.astype(np.float64) - v["density64"]).max()) if c["V"] else 0.0
    assert err_d <= TOL_REL_MAX * max(dmax, 1e-30), (err_d, dmax)
    w = v["density64"] > 1e-3 * dmax
    if w.any():
        err_c = float(np.abs(g.color.astype(np.float64)[w] - v["color64"][w]).max())
        assert err_c <= 1e-4, err_c
    ref.close()
    return g, c


def test_pytest_cloud(vox_ctx, oracle_mod):
    # pytests/test_pipelines.py:313-336 / :497-506: element_count > 0 at voxel 1/8
    cloud = W.pytest_cloud()
    g, c = _check(vox_ctx, oracle_mod, cloud, 1.0 / 8.0)
    assert c["V"] > 0 and g.header["grid_bytes"] > 0


@pytest.mark.parametrize("n,seed", [(1, 0), (7, 1), (200, 2), (5000, 3)])
def test_plain_small(vox_ctx, oracle_mod, n, seed):
    _check(vox_ctx, oracle_mod, W.plain_cloud(n, seed), 0.01)


def test_cluster_small(vox_ctx, oracle_mod):
    _check(vox_ctx, oracle_mod, W.cluster_cloud(20_000, 4, clusters=8), 0.002)


def test_plain_100k(vox_ctx, oracle_mod):
    # the 100k-Gaussian workload at voxel 0.01, in full
    _check(vox_ctx, oracle_mod, W.plain_cloud(100_000, 0), 0.01)


def test_empty_cloud(vox_ctx):
    z = np.zeros((0, 3), np.float32)
    g = vox_ctx.voxelize_host(z, np.zeros((0, 4), np.float32), z, np.zeros(0, np.float32), z, 0.01)
    assert g.counts["voxels"] == 0 and g.counts["pairs"] == 0
    assert g.value_count == 2


def test_transparent_gaussians_emit_nothing(vox_ctx, oracle_mod):
    cloud = W.plain_cloud(64, 5)
    cloud["opacities"][:] = 0.009  # below the 0.01 cutoff of gaussian_prim.slang:65
    g = vox_ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"], 0.01)
    assert g.counts["pairs"] == 0


def test_out_of_range_rejected(vox_ctx):
    from nanovdb_editor.exceptions import PipelineError

    cloud = W.plain_cloud(16, 6)
    cloud["means"][0] = [700.0, 0.0, 0.0]  # 70000 voxels at 0.01 > 65535
    with pytest.raises(PipelineError):
        vox_ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"], 0.01)
    # the context stays usable
    ok = W.plain_cloud(16, 7)
    g = vox_ctx.voxelize_host(ok["means"], ok["quats"], ok["scales"], ok["opacities"], ok["colors"], 0.01)
    assert g.counts["voxels"] > 0


def test_cull_scale_parameter(vox_ctx, oracle_mod):
    cloud = W.plain_cloud(2000, 8)
    _check(vox_ctx, oracle_mod, cloud, 0.01, cull=0.02)


def test_far_from_origin(vox_ctx, oracle_mod):
    # coordinates near the root-key limit: v * vs rounds coarsely in float
    cloud = W.plain_cloud(3000, 9)
    cloud["means"] += np.float32(640.0)
    _check(vox_ctx, oracle_mod, cloud, 0.01)


def test_needles_and_discs(vox_ctx, oracle_mod):
    cloud = W.plain_cloud(3000, 10)
    cloud["scales"][:1000, 0] *= 40.0  # needles
    cloud["scales"][1000:2000, :2] *= 15.0  # discs
    cloud["scales"][2000:, :] *= 0.05  # below the voxel/8 clamp
    _check(vox_ctx, oracle_mod, cloud, 0.01)


def test_leaf_bound_never_skips_a_passing_voxel(oracle_mod):
    """VOX_CHECK_EMIT=1 also walks every bbox leaf the conservative leaf test
    culls and fails the call if one of its voxels passes the reference test."""
    import os

    from nanovdb_editor.vox import VoxContext

    os.environ["VOX_CHECK_EMIT"] = "1"
    try:
        ctx = VoxContext(0)
    finally:
        del os.environ["VOX_CHECK_EMIT"]
    try:
        clouds = [
            (W.plain_cloud(20_000, 12), 0.01),
            (W.cluster_cloud(50_000, 13, clusters=16), 0.002),
            (W.pytest_cloud(), 1.0 / 8.0),
        ]
        far = W.plain_cloud(5000, 14)
        far["means"] -= np.float32(600.0)
        clouds.append((far, 0.01))
        needles = W.plain_cloud(5000, 15)
        needles["scales"][:, 2] *= 20.0
        clouds.append((needles, 0.01))
        # the 2M-Gaussian / 64-cluster cloud at vs 0.002 (about 1.6e9 pairs): the
        # check also runs the reference test on every voxel the linear
        # classification decided and on every pair's RGBA8 byte decided from the
        # float channel's alpha
        clouds.append((W.cluster_cloud(2_000_000, 1, clusters=64), 0.002))
        for cloud, vs in clouds:
            g = ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"], vs)
            assert g.counts["pairs"] > 0
    finally:
        ctx.close()


@pytest.mark.parametrize("make,vs", [
    (lambda: W.plain_cloud(100_000, 0), 0.01),      # the 100k workload: 12 fragment windows
    (lambda: W.plain_cloud(270_000, 21), 0.02),     # two 256K-Gaussian batches
    (lambda: W.pytest_cloud(), 1.0 / 8.0),          # one window
])
def test_reference_window_order(vox_ctx, oracle_mod, make, vs):
    """VOX_FLAG_WINDOW_ORDER: node_idx, node2 addresses and value indices follow
    the reference's 256K-Gaussian x 8M-fragment window build, byte for byte
    against the oracle's window-by-window restatement."""
    from nanovdb_editor.vox import FLAG_WINDOW_ORDER

    cloud = make()
    g = vox_ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"], vs,
                              0.05, flags=FLAG_WINDOW_ORDER)
    ref = oracle_mod.OracleResult(cloud, vs, 0.05, window_mode=1)
    assert ref.counts["error"] == 0
    assert int(g.header["node_order"]) == 1
    n2 = ref.node2()
    if not np.array_equal(g.node2, n2):
        bad = np.nonzero(g.node2.view(np.uint64) != n2.view(np.uint64))[0] if g.node2.shape == n2.shape else []
        pytest.fail(f"node2 differs (windows {ref.counts['windows']}): {len(bad)} words, first {bad[:8]}")
    v = ref.values()
    np.testing.assert_array_equal(g.rgba8, v["rgba8"])
    np.testing.assert_array_equal(g.density, v["density"])
    np.testing.assert_array_equal(g.color, v["color"])
    k_ref, i_ref = ref.pairs()
    k_got, i_got = vox_ctx.pairs()
    np.testing.assert_array_equal(k_got, k_ref)
    np.testing.assert_array_equal(i_got, i_ref)
    ref.close()
