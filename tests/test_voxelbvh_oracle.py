"""VoxelBVH Gaussian ingestion on the CPU (raster/VoxelBVH.cpp:1225-1435).

1. The oracle's restatement against the reference's own shader,
   raster/shaders/voxelbvh/voxelbvh_gaussians_to_ijkl.slang, compiled as C++
   into oracle/_ref/libref_shaders.so (oracle/ref_shaders/build_ref.sh): the
   same keys and Gaussian ids once both are sorted stably by key, for plain,
   clustered, anisotropic, faint and the 32-Gaussian pytest clouds, three
   resolutions, with and without a transform.
2. The range headers against the reference's own
   voxelbvh_find_range_starts.slang and voxelbvh_scatter_range_headers.slang
   (compiled the same way) on the oracle's sorted keys, and the invariants
   they state: ranges partition the sorted keys, one range per distinct key,
   zeros after.
3. The library's host-side transform inverse (no GPU needed).
"""

import ctypes
import os

import numpy as np
import pytest

from nanovdb_editor import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_shaders.so")
LIB = os.path.join(ROOT, "nanovdb-editor_b200", "nanovdb_editor", "lib", "libpnanovdbcompute.so")
SENTINEL = np.uint64(0xFFFFFFFFFFFFFFFF)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("reference shaders not built (oracle/ref_shaders/build_ref.sh needs the reference checkout)")
    L = ctypes.CDLL(REF)
    if not hasattr(L, "ref_voxelbvh_to_ijkl"):
        pytest.skip("oracle/_ref predates the VoxelBVH shader; rerun oracle/ref_shaders/build_ref.sh")
    L.ref_voxelbvh_to_ijkl.argtypes = [ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 9
    if hasattr(L, "ref_voxelbvh_ranges"):
        L.ref_voxelbvh_ranges.argtypes = [ctypes.c_uint32] + [ctypes.c_void_p] * 4
    return L


def transform_4x4():
    """A rotation about z by 0.7 rad, uniform scale 1.5 and a translation, in
    the reference's row-vector convention (translation in the last row)."""
    ang = 0.7
    T = np.eye(4)
    T[:3, :3] = np.array([[np.cos(ang), np.sin(ang), 0], [-np.sin(ang), np.cos(ang), 0], [0, 0, 1]]) * 1.5
    T[3, :3] = [0.3, -2.0, 5.0]
    return T.astype(np.float32)


def inverse_f32(T):
    return np.linalg.inv(T.astype(np.float64)).astype(np.float32)


def clouds():
    faint = W.plain_cloud(300, 31)
    faint["opacities"][::3] = 0.005  # below the 0.01 cut-off: local scale 0
    aniso = W.plain_cloud(300, 32)
    aniso["scales"][:, 0] *= 30.0
    return {
        "plain": W.plain_cloud(600, 21),
        "clusters": W.cluster_cloud(600, 22, clusters=4),
        "pytest32": W.pytest_cloud(),
        "faint": faint,
        "aniso": aniso,
    }


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def ref_keys(L, cloud, res, T, Ti, box):
    n = cloud.n
    pad = 8 * 256 * ((n + 255) // 256)
    k = np.zeros(pad, np.uint64)
    i = np.zeros(pad, np.uint32)
    m, q, s, o = (_f(cloud[x]) for x in ("means", "quats", "scales", "opacities"))
    Tp = None if T is None else _f(T).reshape(16)
    Tip = None if Ti is None else _f(Ti).reshape(16)
    L.ref_voxelbvh_to_ijkl(n, res, m.ctypes.data, o.ctypes.data, q.ctypes.data, s.ctypes.data,
                           None if Tp is None else Tp.ctypes.data, None if Tip is None else Tip.ctypes.data,
                           _f(box).ctypes.data, k.ctypes.data, i.ctypes.data)
    k, i = k[: 8 * n], i[: 8 * n]
    order = np.argsort(k, kind="stable")
    return k[order], i[order]


def check_ranges(keys, rng, count):
    """The reference's header layout for sorted keys."""
    N = keys.size
    starts = np.flatnonzero(np.concatenate([[True], keys[1:] != keys[:-1]])) if N else np.zeros(0, np.int64)
    assert count == starts.size
    ends = np.concatenate([starts[1:], [N]]) if N else starts
    h = rng.reshape(-1, 2)
    np.testing.assert_array_equal(h[:count, 0], starts.astype(np.uint32))
    np.testing.assert_array_equal(h[:count, 1], ends.astype(np.uint32))
    assert not h[count:].any()


@pytest.mark.parametrize("name", ["plain", "clusters", "pytest32", "faint", "aniso"])
@pytest.mark.parametrize("res", [64, 1024, 4096])
@pytest.mark.parametrize("xform", [False, True])
def test_oracle_matches_reference_shader(ref, oracle_mod, name, res, xform):
    cloud = clouds()[name]
    T = transform_4x4() if xform else None
    Ti = inverse_f32(T) if xform else None
    out = oracle_mod.voxelbvh_ijkl(cloud, res, T, Ti)
    assert out["ranges"] > 0
    k, i = ref_keys(ref, cloud, res, T, Ti, out["world_bbox"])
    np.testing.assert_array_equal(out["ijkl"], k)
    np.testing.assert_array_equal(out["prim_id"], i)


@pytest.mark.parametrize("name", ["plain", "clusters", "faint"])
@pytest.mark.parametrize("res", [64, 4096])
def test_oracle_ranges_match_reference_shaders(ref, oracle_mod, name, res):
    # voxelbvh_find_range_starts + the inclusive global_scan +
    # voxelbvh_scatter_range_headers, compiled from the reference, on the
    # oracle's sorted keys
    if not hasattr(ref, "ref_voxelbvh_ranges"):
        pytest.skip("oracle/_ref predates the range shaders; rerun oracle/ref_shaders/build_ref.sh")
    out = oracle_mod.voxelbvh_ijkl(clouds()[name], res)
    keys = np.ascontiguousarray(out["ijkl"])
    N = keys.size
    starts, scan = np.zeros(N, np.uint32), np.zeros(N, np.uint32)
    headers = np.full(2 * N, 0xDEADBEEF, np.uint32)
    ref.ref_voxelbvh_ranges(N, keys.ctypes.data, starts.ctypes.data, scan.ctypes.data, headers.ctypes.data)
    np.testing.assert_array_equal(headers, out["range"])
    assert int(scan[-1]) == out["ranges"]


@pytest.mark.parametrize("res", [16, 1024])
def test_oracle_invariants(oracle_mod, res):
    cloud = W.cluster_cloud(2000, 41, clusters=6)
    out = oracle_mod.voxelbvh_ijkl(cloud, res)
    keys, ids = out["ijkl"], out["prim_id"]
    n = cloud.n
    assert np.all(keys[1:] >= keys[:-1])
    real = keys != SENTINEL
    # every Gaussian has 1..8 cells, all on one level in 0..11
    per = np.bincount(ids[real].astype(np.int64), minlength=n)
    assert per.min() >= 1 and per.max() <= 8
    lv = (keys[real] & np.uint64(0xFFFF)).astype(np.int64)
    assert lv.max() <= 11
    lv_of = np.full(n, -1)
    lv_of[ids[real]] = lv
    assert np.all(lv_of[ids[real]] == lv)
    # sentinels carry the invalid id; ids ascend within a key (stable sort)
    assert np.all(ids[~real] == 0xFFFFFFFF)
    check_ranges(keys, out["range"], out["ranges"])
    same = (keys[1:] == keys[:-1]) & real[1:]
    assert np.all(ids[1:][same] > ids[:-1][same])
    # the world box encloses every mean
    box = out["world_bbox"]
    m = cloud["means"]
    assert np.all(m >= box[:3]) and np.all(m <= box[3:])


def test_oracle_thread_count_independent(oracle_mod):
    # the world box is a total-order min / max and every Gaussian owns its
    # 8 slots, so splitting the Gaussians over threads changes nothing
    cloud = W.cluster_cloud(5000, 42, clusters=8)
    one = oracle_mod.voxelbvh_ijkl(cloud, 1024, nthreads=1)
    for t in (2, 7):
        many = oracle_mod.voxelbvh_ijkl(cloud, 1024, nthreads=t)
        assert many["ranges"] == one["ranges"]
        for k in ("ijkl", "prim_id", "range", "world_bbox"):
            np.testing.assert_array_equal(many[k], one[k])


def test_oracle_rejects_unbounded_cells(oracle_mod):
    cloud = W.plain_cloud(50, 43)
    cloud["means"][7, 1] = np.nan
    assert oracle_mod.voxelbvh_ijkl(cloud, 256)["ranges"] == -1


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import build_ext

        build_ext.build()
    L = ctypes.CDLL(LIB)
    L.vox_voxelbvh_transform_inverse.restype = ctypes.c_int
    L.vox_voxelbvh_transform_inverse.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    return L


def test_transform_inverse_host(lib):
    T = transform_4x4()
    inv = np.empty(16, np.float32)
    assert lib.vox_voxelbvh_transform_inverse(_f(T).ctypes.data, inv.ctypes.data) == 0
    ref = np.linalg.inv(T.astype(np.float64))
    np.testing.assert_allclose(inv.reshape(4, 4), ref, rtol=0, atol=1e-6)
    # correctly rounded from double for this well-conditioned matrix
    assert np.max(np.abs(inv.reshape(4, 4).astype(np.float64) - ref)) <= np.max(np.abs(ref)) * 2.0 ** -23
    sing = np.eye(4, dtype=np.float32)
    sing[2, 2] = 0.0
    assert lib.vox_voxelbvh_transform_inverse(sing.ctypes.data, inv.ctypes.data) == -1
    bad = np.eye(4, dtype=np.float32)
    bad[0, 1] = np.inf
    assert lib.vox_voxelbvh_transform_inverse(bad.ctypes.data, inv.ctypes.data) == -1
