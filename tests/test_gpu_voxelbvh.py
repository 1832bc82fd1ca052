"""VoxelBVH Gaussian ingestion on the GPU (vox_voxelbvh_ijkl_from_gaussians,
replacing ijkl_from_gaussians of raster/VoxelBVH.cpp:1225-1435) against the
CPU oracle: sorted keys, Gaussian ids, range headers and the world box, bit
for bit.  With a transform, the oracle is given the inverse the library
applies (vox_voxelbvh_transform_inverse)."""

import numpy as np
import pytest

from nanovdb_editor import workloads as W

pytestmark = pytest.mark.gpu

SENTINEL = np.uint64(0xFFFFFFFFFFFFFFFF)


def _dev(cloud):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(cloud[k], dtype=np.float32)).cuda()
            for k in ("means", "opacities", "quats", "scales")]


def _run(vox_ctx, cloud, res, T=None):
    m, o, q, s = _dev(cloud)
    out = vox_ctx.voxelbvh_ijkl_from_gaussians(m, o, q, s, res, T)
    return {
        "ijkl": out["ijkl"].cpu().numpy().view(np.uint64),
        "prim_id": out["prim_id"].cpu().numpy().view(np.uint32),
        "range": out["range"].cpu().numpy().view(np.uint32),
        "world_bbox": out["world_bbox"].cpu().numpy(),
        "range_count": out["range_count"],
    }


def _compare(got, ref):
    np.testing.assert_array_equal(got["world_bbox"].view(np.uint32), ref["world_bbox"].view(np.uint32))
    np.testing.assert_array_equal(got["ijkl"], ref["ijkl"])
    np.testing.assert_array_equal(got["prim_id"], ref["prim_id"])
    np.testing.assert_array_equal(got["range"], ref["range"])
    assert got["range_count"] == ref["ranges"]


def _transform():
    ang = 0.7
    T = np.eye(4)
    T[:3, :3] = np.array([[np.cos(ang), np.sin(ang), 0], [-np.sin(ang), np.cos(ang), 0], [0, 0, 1]]) * 1.5
    T[3, :3] = [0.3, -2.0, 5.0]
    return T.astype(np.float32)


def _clouds():
    faint = W.plain_cloud(3000, 31)
    faint["opacities"][::3] = 0.005
    aniso = W.plain_cloud(3000, 32)
    aniso["scales"][:, 0] *= 30.0
    return {
        "plain": W.plain_cloud(20_000, 21),
        "clusters": W.cluster_cloud(20_000, 22, clusters=16),
        "pytest32": W.pytest_cloud(),
        "faint": faint,
        "aniso": aniso,
    }


@pytest.mark.parametrize("name", ["plain", "clusters", "pytest32", "faint", "aniso"])
@pytest.mark.parametrize("res", [64, 1024, 4096])
def test_ijkl_matches_oracle(vox_ctx, oracle_mod, name, res):
    cloud = _clouds()[name]
    _compare(_run(vox_ctx, cloud, res), oracle_mod.voxelbvh_ijkl(cloud, res))


@pytest.mark.parametrize("res", [256, 4096])
def test_ijkl_with_transform_matches_oracle(vox_ctx, oracle_mod, res):
    cloud = W.cluster_cloud(10_000, 23, clusters=8)
    T = _transform()
    Ti = vox_ctx.voxelbvh_transform_inverse(T)
    _compare(_run(vox_ctx, cloud, res, T), oracle_mod.voxelbvh_ijkl(cloud, res, T, Ti))


@pytest.mark.parametrize("n", [1, 2, 255, 256, 257])
def test_ijkl_small_counts(vox_ctx, oracle_mod, n):
    cloud = W.plain_cloud(n, 100 + n)
    _compare(_run(vox_ctx, cloud, 512), oracle_mod.voxelbvh_ijkl(cloud, 512))


def test_ijkl_empty(vox_ctx, oracle_mod):
    cloud = W.plain_cloud(0, 7)
    got = _run(vox_ctx, cloud, 512)
    ref = oracle_mod.voxelbvh_ijkl(cloud, 512)
    assert got["ijkl"].size == 0 and got["range_count"] == 0 == ref["ranges"]
    np.testing.assert_array_equal(got["world_bbox"].view(np.uint32), ref["world_bbox"].view(np.uint32))


def test_ijkl_large_properties(vox_ctx, oracle_mod):
    # 400k Gaussians (3.2M keys, above the 126 MB L2 with the sort's buffers):
    # exact against the oracle, and the sort / range invariants
    cloud = W.cluster_cloud(400_000, 24, clusters=64)
    got = _run(vox_ctx, cloud, 4096)
    ref = oracle_mod.voxelbvh_ijkl(cloud, 4096)
    _compare(got, ref)
    k = got["ijkl"]
    assert np.all(k[1:] >= k[:-1])
    real = k != SENTINEL
    assert np.bincount(got["prim_id"][real].astype(np.int64), minlength=cloud.n).max() <= 8


def test_ijkl_full_key_sort_path(vox_ctx, oracle_mod, monkeypatch):
    # the 64-bit key sort (taken when a cell lies outside [0, 2^15)) gives
    # the same result as the compressed-key sort
    cloud = W.cluster_cloud(30_000, 25, clusters=8)
    ref = oracle_mod.voxelbvh_ijkl(cloud, 4096)
    monkeypatch.setenv("VOX_VB_SORT64", "1")
    got = _run(vox_ctx, cloud, 4096)
    assert vox_ctx.stats()["vb_sort_bits"] == 64
    _compare(got, ref)
    monkeypatch.delenv("VOX_VB_SORT64")
    got = _run(vox_ctx, cloud, 4096)
    assert vox_ctx.stats()["vb_sort_bits"] < 64
    _compare(got, ref)


def test_ijkl_far_cloud_without_cells(vox_ctx, oracle_mod):
    # 3e8 from the origin the float cell lattice is coarser than the cloud:
    # no Gaussian overlaps a cell, every slot is unused (one range), and the
    # sort is skipped (unused slots are already in order)
    cloud = W.plain_cloud(2000, 60)
    cloud["means"][:, 0] += np.float32(3e8)
    ref = oracle_mod.voxelbvh_ijkl(cloud, 4096)
    assert ref["ranges"] == 1 and np.all(ref["ijkl"] == SENTINEL)
    _compare(_run(vox_ctx, cloud, 4096), ref)


@pytest.mark.parametrize("offset", [1e6, 1e7])
def test_ijkl_far_cloud(vox_ctx, oracle_mod, offset):
    # far from the origin the cell arithmetic rounds coarsely; still bit-exact
    cloud = W.plain_cloud(2000, 60)
    cloud["means"][:, 0] += np.float32(offset)
    _compare(_run(vox_ctx, cloud, 4096), oracle_mod.voxelbvh_ijkl(cloud, 4096))


def test_ijkl_signed_zero_world_min(vox_ctx, oracle_mod):
    # a faint Gaussian (opacity < 0.01: a point box) at x = -0 is the world
    # minimum in x: its corners are +0 and -0, and -0 orders first
    cloud = W.plain_cloud(200, 50)
    cloud["means"][:, 0] = np.abs(cloud["means"][:, 0]) + 0.5
    cloud["means"][3] = [-0.0, 0.1, 0.1]
    cloud["opacities"][3] = 0.005
    ref = oracle_mod.voxelbvh_ijkl(cloud, 256)
    assert ref["world_bbox"].view(np.uint32)[0] == 0x80000000
    _compare(_run(vox_ctx, cloud, 256), ref)


@pytest.mark.parametrize("value", [np.nan, np.inf, 1e30])
def test_ijkl_rejects_non_finite_and_recovers(vox_ctx, oracle_mod, value):
    # a non-finite box corner (NaN / inf mean), or a finite box beyond
    # +-65536 voxels (a far-away Gaussian next to a small cloud is fine: the
    # cloud's cells shrink), is reported, and the context keeps working
    from nanovdb_editor.exceptions import PipelineError

    bad = W.plain_cloud(1000, 44)
    bad["means"][17, 0] = value
    if value == 1e30:
        ref = oracle_mod.voxelbvh_ijkl(bad, 512)
        assert ref["ranges"] > 0
        _compare(_run(vox_ctx, bad, 512), ref)
    else:
        assert oracle_mod.voxelbvh_ijkl(bad, 512)["ranges"] == -1
        with pytest.raises(PipelineError, match="outside"):
            _run(vox_ctx, bad, 512)
    good = W.plain_cloud(1000, 45)
    _compare(_run(vox_ctx, good, 512), oracle_mod.voxelbvh_ijkl(good, 512))


def test_ijkl_argument_checks(vox_ctx):
    from nanovdb_editor.exceptions import PipelineError

    cloud = W.plain_cloud(10, 46)
    with pytest.raises(PipelineError):
        _run(vox_ctx, cloud, 0)
    with pytest.raises(PipelineError):
        _run(vox_ctx, cloud, 4097)
    sing = np.eye(4, dtype=np.float32)
    sing[1, 1] = 0.0
    with pytest.raises(PipelineError):
        _run(vox_ctx, cloud, 256, sing)


@pytest.mark.parametrize("fmt", ["npz", "ply"])
def test_ijkl_from_file(vox_ctx, oracle_mod, tmp_path, fmt):
    # ijkl_from_gaussians_file: raw attributes in a file, activated on the
    # host (the raster path's preprocessing restated by the oracle)
    from test_gpu_dropin import _write_ply

    raw = W.cluster_cloud(5000, 47, clusters=4).raw_arrays()
    path = tmp_path / f"splats.{fmt}"
    if fmt == "npz":
        np.savez(path, means=raw[0], opacities=raw[1], quaternions=raw[2], scales=raw[3], sh_0=raw[4], sh_n=raw[5])
    else:
        _write_ply(path, raw)
    got = vox_ctx.voxelbvh_ijkl_from_file(str(path), 512)
    act = oracle_mod.preprocess(raw)
    np.testing.assert_array_equal(got["quaternions"].reshape(-1, 4).view(np.uint32), act["quats"].view(np.uint32))
    np.testing.assert_array_equal(got["scales"].reshape(-1, 3).view(np.uint32), act["scales"].view(np.uint32))
    np.testing.assert_array_equal(got["opacities"].view(np.uint32), act["opacities"].view(np.uint32))
    ref = oracle_mod.voxelbvh_ijkl(act, 512)
    np.testing.assert_array_equal(got["world_bbox"].view(np.uint32), ref["world_bbox"].view(np.uint32))
    np.testing.assert_array_equal(got["ijkl"], ref["ijkl"])
    np.testing.assert_array_equal(got["prim_id"], ref["prim_id"])
    np.testing.assert_array_equal(got["range"], ref["range"])
