"""The CPU oracle against golden fixtures made from the reference itself
(tests/golden/make_golden.py: the reference's shader files compiled as C++),
so the pin holds where the reference checkout is absent.

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
    assert len(_files("raster_")) >= 5 and len(_files("voxelbvh_")) >= 4


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
