"""The CPU oracle against golden fixtures made from the reference itself
(tests/golden/make_golden.py: the reference's shader files compiled as C++),
so the pin holds where the reference checkout is absent.

topology_*.npz: the node2 region, node counts, value count and bbox the
reference's grid-build shaders produce (grid_build_*.slang, run window by
window as raster_gaussian_3d runs them), including a 12-window and a
two-prim-batch cloud.

raster_*.npz: per-Gaussian bbox and fragment count (gaussian_prim.slang),
the sorted passing (voxel, Gaussian) pairs of one fragment window
(fanout_*.slang, gaussian_frag_alloc.slang) and the per-voxel RGBA8 maximum
(gaussian_frag_color.slang).  voxelbvh_*.npz: sorted keys and ids
(voxelbvh_gaussians_to_ijkl.slang) and range headers
(voxelbvh_find_range_starts.slang, voxelbvh_scatter_range_headers.slang).
"""

import glob
import os

import numpy as np
import pytest

from nanovdb_editor import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cloud(z):
    c = W.GaussianCloud()
    for k in ("means", "quats", "scales", "opacities"):
        c[k] = np.array(z[k])
    c["colors"] = np.array(z["colors"]) if "colors" in z else np.full((c.n, 3), 0.5, np.float32)
    return c


def _files(prefix):
    return sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


def test_fixtures_present():
    assert len(_files("raster_")) >= 5 and len(_files("voxelbvh_")) >= 4 and len(_files("topology_")) >= 7


@pytest.mark.parametrize("path", _files("raster_"), ids=os.path.basename)
def test_oracle_matches_golden_raster(oracle_mod, path):
    z = np.load(path)
    cloud = _cloud(z)
    vs, cull = float(z["voxel_size"]), float(z["cull"])
    L = oracle_mod.lib()
    for g in range(cloud.n):
        b = np.zeros(6, np.int32)
        fp = np.zeros(1, np.uint64)
        valid = L.ov_prim_bbox(np.ascontiguousarray(cloud["means"][g]).ctypes.data,
                               np.ascontiguousarray(cloud["quats"][g]).ctypes.data,
                               np.ascontiguousarray(cloud["scales"][g]).ctypes.data,
                               float(cloud["opacities"][g]), vs, b.ctypes.data, fp.ctypes.data)
        assert valid == 1
        np.testing.assert_array_equal(b, z["bbox"][g])
        assert int(fp[0]) == int(z["counts"][g])
    res = oracle_mod.OracleResult(cloud, vs, cull, window_mode=1, nthreads=2)
    k, i = res.pairs()
    np.testing.assert_array_equal(k, z["pair_keys"])
    np.testing.assert_array_equal(i, z["pair_ids"])
    vox_ijk, vidx = res.voxels()
    vk = np.array([oracle_mod.hier_key(*x) for x in vox_ijk], dtype=np.uint64)
    order = np.argsort(vk)
    np.testing.assert_array_equal(vk[order], z["voxel_keys"])
    np.testing.assert_array_equal(res.values()["rgba8"][vidx[order]], z["voxel_rgba"])
    res.close()


@pytest.mark.parametrize("path", _files("voxelbvh_"), ids=os.path.basename)
def test_oracle_matches_golden_voxelbvh(oracle_mod, path):
    z = np.load(path)
    T = np.array(z["transform"]) if "transform" in z else None
    Ti = np.array(z["transform_inv"]) if "transform_inv" in z else None
    out = oracle_mod.voxelbvh_ijkl(_cloud(z), int(z["resolution"]), T, Ti, nthreads=2)
    np.testing.assert_array_equal(out["world_bbox"].view(np.uint32), z["world_bbox"].view(np.uint32))
    np.testing.assert_array_equal(out["ijkl"], z["ijkl"])
    np.testing.assert_array_equal(out["prim_id"], z["prim_id"])
    np.testing.assert_array_equal(out["range"], z["range"])
    assert out["ranges"] == int(z["ranges"])


def topology_cloud(z):
    """The fixture's cloud: its float32 inputs, or its generator re-run and
    checked against the SHA-256 of the inputs it was made from."""
    import hashlib

    if "means" in z:
        return _cloud(z)
    gen = getattr(W, str(z["generator"]))
    c = gen(int(z["count"]), int(z["seed"]))
    h = hashlib.sha256()
    for k in ("means", "quats", "scales", "opacities"):
        h.update(np.ascontiguousarray(c[k], np.float32).tobytes())
    assert h.hexdigest() == str(z["inputs_sha256"]), "the generator no longer reproduces the fixture's inputs"
    return c


def check_topology(z, region, counts, bbox):
    """A node2 region, node counts and bbox against a topology fixture."""
    import hashlib

    assert counts == {k: int(z[k]) for k in ("upper", "lower", "leaf", "value_count")}
    np.testing.assert_array_equal(np.asarray(bbox, np.int32), z["bbox"])
    assert region.size == int(z["node2_bytes"])
    if "node2" in z:
        np.testing.assert_array_equal(region, z["node2"])
    assert hashlib.sha256(region.tobytes()).hexdigest() == str(z["node2_sha256"])


@pytest.mark.parametrize("path", _files("topology_"), ids=os.path.basename)
def test_oracle_matches_golden_topology(oracle_mod, path):
    """The oracle's window-by-window node2 build (window_mode 1) against the
    region the reference's grid-build shaders wrote for the same cloud:
    raster_gaussian_3d's prim batches of 256K and fragment windows of 8M
    (raster/Raster.cpp:420-510), per window and tree level
    grid_build_set_masks / count_new / scatter_new / finalize
    (raster/GridBuild.cpp:361-506), then grid_build_blindmetadata and
    grid_build_compute_bbox (GridBuild.cpp:508-650)."""
    z = np.load(path)
    cloud = topology_cloud(z)
    res = oracle_mod.OracleResult(cloud, float(z["voxel_size"]), 0.05, window_mode=1)
    assert res.counts["windows"] == int(z["windows"])
    check_topology(z, res.node2(), {k: res.counts[k] for k in ("upper", "lower", "leaf", "value_count")}, res.bbox())
    res.close()
