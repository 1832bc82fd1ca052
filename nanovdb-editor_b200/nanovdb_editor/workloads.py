"""Seeded synthetic Gaussian clouds for the voxelization path.

The reference ships no benchmark data for raster3d (its sample ``data/splats.npz``
is not distributed), so these generators stand in for it with the shapes and
value distributions the workload definitions name:

* ``plain_cloud``      100k Gaussians, means U[-1,1]^3, per-axis scales
                       exp(N(ln 0.01, 0.3)), uniform unit quaternions, opacity
                       U[0.05, 1], RGB U[0, 1]; voxel size 0.01.
* ``cluster_cloud``    Gaussians drawn from surface-like clusters: centres
                       U[-1,1]^3, members spread on a random plane with sigma 0.1
                       in-plane and 0.005 along the normal, per-axis scales
                       exp(N(ln 0.003, 0.5)) with anisotropy capped at 20:1.
                       2M Gaussians at voxel 0.002 is the at-scale workload.
* ``batch_clouds``     uneven batches: log-uniform cloud sizes and voxel sizes,
                       1-16 clusters per cloud (256 clouds of 1k-200k Gaussians
                       at voxel 0.002-0.02 is the batched workload).
* ``pytest_cloud``     the 32-Gaussian cloud of the reference's pipeline test
                       (means N(0, 0.3), opacity logit 0.9, identity quaternions,
                       log-scale -3, SH0 0.5) at voxel 1/8.

Every generator returns activated attributes (the inputs of ``raster_to_nanovdb``)
and ``raw_arrays()`` turns them into the on-disk convention consumed by
``raster_to_nanovdb_from_arrays`` (log scales, logit opacities, SH0 colour).
"""

from __future__ import annotations

import numpy as np

SH_C0 = 0.28209479177387814


class GaussianCloud(dict):
    """means (N,3), quats (N,4 w,x,y,z), scales (N,3), colors (N,3), opacities (N,) float32."""

    @property
    def n(self) -> int:
        return int(self["means"].shape[0])

    def raw_arrays(self):
        """[means, opacity logits, quats, log scales, sh_0, sh_n] in the reference's canonical order."""
        op = np.clip(self["opacities"].astype(np.float64), 1e-7, 1 - 1e-7)
        logit = np.log(op / (1.0 - op)).astype(np.float32)
        log_s = np.log(self["scales"].astype(np.float64)).astype(np.float32)
        sh0 = ((self["colors"].astype(np.float64) - 0.5) / SH_C0).astype(np.float32)
        return [
            np.ascontiguousarray(self["means"], dtype=np.float32),
            np.ascontiguousarray(logit, dtype=np.float32),
            np.ascontiguousarray(self["quats"], dtype=np.float32),
            np.ascontiguousarray(log_s, dtype=np.float32),
            np.ascontiguousarray(sh0, dtype=np.float32),
            np.zeros(0, dtype=np.float32),
        ]


def _unit_quats(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


def plain_cloud(n: int = 100_000, seed: int = 0) -> GaussianCloud:
    rng = np.random.default_rng(seed)
    means = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    scales = np.exp(rng.normal(np.log(0.01), 0.3, (n, 3))).astype(np.float32)
    quats = _unit_quats(rng, n)
    opac = rng.uniform(0.05, 1.0, n).astype(np.float32)
    colors = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    return GaussianCloud(means=means, quats=quats, scales=scales, colors=colors, opacities=opac)


def cluster_cloud(
    n: int = 2_000_000,
    seed: int = 1,
    clusters: int = 64,
    scale_mu: float = 0.003,
    scale_sigma: float = 0.5,
    in_plane: float = 0.1,
    normal: float = 0.005,
    max_aniso: float = 20.0,
) -> GaussianCloud:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-1.0, 1.0, (clusters, 3))
    normals = rng.standard_normal((clusters, 3))
    normals /= np.linalg.norm(normals, axis=1, keepdims=True)
    # two in-plane axes per cluster
    helper = np.where(np.abs(normals[:, :1]) < 0.9, np.array([[1.0, 0.0, 0.0]]), np.array([[0.0, 1.0, 0.0]]))
    u = np.cross(normals, helper)
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(normals, u)
    cid = rng.integers(0, clusters, n)
    a = rng.normal(0.0, in_plane, n)
    b = rng.normal(0.0, in_plane, n)
    c = rng.normal(0.0, normal, n)
    means = centres[cid] + a[:, None] * u[cid] + b[:, None] * v[cid] + c[:, None] * normals[cid]
    scales = np.exp(rng.normal(np.log(scale_mu), scale_sigma, (n, 3)))
    smax = scales.max(axis=1, keepdims=True)
    scales = np.maximum(scales, smax / max_aniso)
    quats = _unit_quats(rng, n)
    opac = rng.uniform(0.05, 1.0, n)
    colors = rng.uniform(0.0, 1.0, (n, 3))
    return GaussianCloud(
        means=means.astype(np.float32),
        quats=quats,
        scales=scales.astype(np.float32),
        colors=colors.astype(np.float32),
        opacities=opac.astype(np.float32),
    )


def pytest_cloud(n: int = 32) -> GaussianCloud:
    """Raw-convention cloud of the reference pipeline test, returned activated."""
    rng = np.random.default_rng(0)
    means = (rng.standard_normal((n, 3)) * 0.3).astype(np.float32)
    logit = np.full(n, 0.9, dtype=np.float32)
    quats = np.tile(np.array([1.0, 0.0, 0.0, 0.0], dtype=np.float32), (n, 1))
    log_s = np.full((n, 3), -3.0, dtype=np.float32)
    sh0 = np.full((n, 3), 0.5, dtype=np.float32)
    return GaussianCloud(
        means=means,
        quats=quats,
        scales=np.exp(log_s.astype(np.float64)).astype(np.float32),
        colors=(SH_C0 * sh0 + 0.5).astype(np.float32),
        opacities=(1.0 / (1.0 + np.exp(-logit.astype(np.float64)))).astype(np.float32),
        raw=[means, logit, quats, log_s, sh0, np.zeros(0, dtype=np.float32)],
    )


def concat(clouds) -> GaussianCloud:
    """One cloud of all clouds' Gaussians, in order."""
    keys = ("means", "quats", "scales", "colors", "opacities")
    return GaussianCloud(**{k: np.ascontiguousarray(np.concatenate([c[k] for c in clouds], axis=0)) for k in keys})


def batch_clouds(count: int = 256, seed: int = 3, min_n: int = 1_000, max_n: int = 200_000,
                 vs_min: float = 0.002, vs_max: float = 0.02, max_clusters: int = 16):
    """Uneven batch: `count` clouds of log-uniform size in [min_n, max_n], each a
    cluster_cloud with 1..max_clusters clusters and its own voxel size,
    log-uniform in [vs_min, vs_max].  Returns (list of clouds, cloud_start int64
    [count + 1], voxel_sizes float32 [count])."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(min_n), np.log(max_n), count)).astype(np.int64)
    clusters = rng.integers(1, max_clusters + 1, count)
    vs = np.exp(rng.uniform(np.log(vs_min), np.log(vs_max), count)).astype(np.float32)
    clouds = [cluster_cloud(int(n), int(seed * 100003 + i), clusters=int(c)) for i, (n, c) in enumerate(zip(sizes, clusters))]
    start = np.zeros(count + 1, dtype=np.int64)
    start[1:] = np.cumsum(sizes)
    return clouds, start, vs


WORKLOADS = {
    "plain_100k_vs0.01": (lambda: plain_cloud(100_000, 0), 0.01),
    "cluster_2M_vs0.002": (lambda: cluster_cloud(2_000_000, 1), 0.002),
    "cluster_500k_vs0.004": (lambda: cluster_cloud(500_000, 2), 0.004),
}
