"""The CUDA path against the golden fixtures made from the reference itself
(tests/golden/make_golden.py: the reference's shaders compiled as C++),
directly rather than through the oracle: the sorted passing (voxel key,
Gaussian) pairs and the multiset of per-voxel RGBA8 maxima of the raster
path, every VoxelBVH ingestion output, and the node2 topology of the
reference's grid-build shaders (topology_*.npz).  (The transformed VoxelBVH
fixture is covered through the oracle, which is given the library's own
transform inverse.)"""

import glob
import os

import numpy as np
import pytest

from nanovdb_editor import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cloud(z):
    c = W.GaussianCloud()
    for k in ("means", "quats", "scales", "opacities"):
        c[k] = np.array(z[k])
    c["colors"] = np.array(z["colors"]) if "colors" in z else np.full((c.n, 3), 0.5, np.float32)
    return c


RASTER = sorted(glob.glob(os.path.join(GOLDEN, "raster_*.npz")))
VOXELBVH = sorted(p for p in glob.glob(os.path.join(GOLDEN, "voxelbvh_*.npz")) if "transform" not in p)


@pytest.mark.parametrize("path", RASTER, ids=os.path.basename)
def test_gpu_matches_golden_raster(vox_ctx, path):
    z = np.load(path)
    cloud = _cloud(z)
    g = vox_ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"],
                              float(z["voxel_size"]), float(z["cull"]))
    k, i = vox_ctx.pairs()
    np.testing.assert_array_equal(k, z["pair_keys"])
    np.testing.assert_array_equal(i, z["pair_ids"])
    assert g.counts["voxels"] == z["voxel_keys"].size
    # value indices 0 and 1 are the background; the voxels follow
    np.testing.assert_array_equal(np.sort(g.rgba8[2:]), np.sort(z["voxel_rgba"]))


@pytest.mark.parametrize("path", VOXELBVH, ids=os.path.basename)
def test_gpu_matches_golden_voxelbvh(vox_ctx, path):
    from test_gpu_voxelbvh import _compare, _run

    z = np.load(path)
    got = _run(vox_ctx, _cloud(z), int(z["resolution"]))
    _compare(got, {"ijkl": z["ijkl"], "prim_id": z["prim_id"], "range": z["range"],
                   "world_bbox": np.array(z["world_bbox"]), "ranges": int(z["ranges"])})


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "topology_*.npz"))), ids=os.path.basename)
def test_gpu_matches_golden_topology(vox_ctx, path):
    """The CUDA path in the reference's node order (VOX_FLAG_WINDOW_ORDER)
    against the node2 region the reference's grid-build shaders produce
    (raster/GridBuild.cpp:361-650 run window by window as
    raster/Raster.cpp:420-510 runs it): every byte of the region, the node
    counts, the value count and the bbox - including the cfg0 cloud of 100K
    Gaussians (12 fragment windows) and a 300K cloud (two prim batches)."""
    from nanovdb_editor.vox import FLAG_WINDOW_ORDER
    from test_golden import check_topology, topology_cloud

    z = np.load(path)
    cloud = topology_cloud(z)
    g = vox_ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"],
                              float(z["voxel_size"]), 0.05, FLAG_WINDOW_ORDER)
    h = g.header
    counts = {"upper": int(h["upper_count"]), "lower": int(h["lower_count"]), "leaf": int(h["leaf_count"]),
              "value_count": int(h["value_count"])}
    check_topology(z, np.array(g.node2), counts, np.array(h["bbox"]))
