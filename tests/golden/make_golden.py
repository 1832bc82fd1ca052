"""Generates the golden fixtures in this folder from the reference itself:
the reference's shader files compiled as C++ into oracle/_ref/libref_shaders.so
by oracle/ref_shaders/build_ref.sh (needs the reference checkout; run where it
exists).  Each fixture holds its float32 inputs and the reference's outputs,
so tests/test_golden.py checks the CPU oracle against them without the
reference.

    python tests/golden/make_golden.py

Fixtures:
  raster_<case>.npz    gaussian_prim bbox + fragment count per Gaussian, the
                       sorted (hierarchical voxel key, Gaussian) pairs that
                       pass gaussian_frag_alloc in one fragment window, and
                       the per-voxel RGBA8 maximum of gaussian_frag_color
  voxelbvh_<case>.npz  voxelbvh_gaussians_to_ijkl keys and ids (sorted
                       stably by key) and the range headers of
                       voxelbvh_find_range_starts / scatter_range_headers
  topology_<case>.npz  the node2 region (root first, every node at its node2
                       maximum size in the order the reference allocates it)
                       that the reference's grid-build shaders produce for the
                       cloud - grid_build_set_masks / count_new / scatter_new /
                       finalize per tree level and fragment window, then
                       grid_build_blindmetadata and grid_build_compute_bbox -
                       as its SHA-256 (and the bytes themselves for the small
                       clouds), with node counts, value count, window count and
                       bbox.  The two large clouds (12 fragment windows; two
                       prim batches) are stored as their generator, seed and
                       the SHA-256 of their float32 inputs instead of the inputs.

    python tests/golden/make_golden.py [--topology]   (--topology: only topology_*)
"""

import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "nanovdb-editor_b200"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import oracle as O  # noqa: E402
from nanovdb_editor import workloads as W  # noqa: E402

P = ctypes.c_void_p


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def load_ref():
    path = O.build_ref()
    if not path:
        raise SystemExit("reference shaders unavailable: oracle/ref_shaders/build_ref.sh needs the reference checkout")
    L = ctypes.CDLL(path)
    L.ref_gaussian_prim.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float] + [P] * 6
    L.ref_fanout.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64] + [P] * 5
    L.ref_frag_alloc.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float] + [P] * 8
    L.ref_frag_color.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_int] + [P] * 9
    L.ref_voxelbvh_to_ijkl.argtypes = [ctypes.c_uint32, ctypes.c_uint32] + [P] * 9
    L.ref_voxelbvh_ranges.argtypes = [ctypes.c_uint32] + [P] * 4
    return L


def raster_cases():
    tiny = W.plain_cloud(60, 23)
    tiny["scales"][:] = 1e-5  # clamped to voxel / 8 (gaussian_prim.slang:67-68)
    aniso = W.plain_cloud(30, 24)
    aniso["scales"][:, 0] *= 20.0
    return {
        "plain": (W.plain_cloud(150, 21), 0.02),
        "clusters": (W.cluster_cloud(150, 22, clusters=3), 0.01),
        "pytest32": (W.pytest_cloud(), 1.0 / 8.0),
        "tiny": (tiny, 0.02),
        "aniso": (aniso, 0.02),
    }


def raster_fixture(L, cloud, vs, cull=0.05):
    n = cloud.n
    m, q, s, o, c = (_f(cloud[k]) for k in ("means", "quats", "scales", "opacities", "colors"))
    counts = np.zeros(n, np.uint64)
    bbox = np.zeros((n, 6), np.int32)
    L.ref_gaussian_prim(n, 0, n, vs, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, counts.ctypes.data, bbox.ctypes.data)
    scan = np.cumsum(counts).astype(np.uint64)
    F = int(scan[-1])
    slots = max(256, (F + 255) // 256 * 256)
    tmp, pidx, ridx = (np.zeros(slots, np.uint32) for _ in range(3))
    L.ref_fanout(n, slots, 0, counts.ctypes.data, scan.ctypes.data, tmp.ctypes.data, pidx.ctypes.data, ridx.ctypes.data)
    ijk = np.full((slots, 3), 0x7FFFFFFF, np.int32)
    L.ref_frag_alloc(slots, 0, vs, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, pidx.ctypes.data, ridx.ctypes.data, bbox.ctypes.data, ijk.ctypes.data)
    rgba = np.zeros(slots, np.uint32)
    L.ref_frag_color(slots, 0, vs, cull, 0, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, c.ctypes.data, pidx.ctypes.data, ridx.ctypes.data, bbox.ctypes.data, rgba.ctypes.data)
    live = (ridx != 0xFFFFFFFF) & (ijk[:, 2] != 0x7FFFFFFF)
    gid, vox, col = pidx[live], ijk[live], rgba[live]
    keys = np.array([O.hier_key(*v) for v in vox], dtype=np.uint64)
    order = np.lexsort((gid, keys))
    # per-voxel maximum of the packed RGBA8 (gaussian_frag_color.slang:239-246)
    vmax = {}
    for k, v in zip(keys.tolist(), col.tolist()):
        vmax[k] = max(vmax.get(k, 0), v)
    vk = np.array(sorted(vmax), dtype=np.uint64)
    return dict(means=m, quats=q, scales=s, opacities=o, colors=c, voxel_size=np.float32(vs), cull=np.float32(cull),
                counts=counts, bbox=bbox, pair_keys=keys[order], pair_ids=gid[order],
                voxel_keys=vk, voxel_rgba=np.array([vmax[k] for k in vk.tolist()], dtype=np.uint32))


def voxelbvh_cases():
    faint = W.plain_cloud(120, 31)
    faint["opacities"][::3] = 0.005
    return {
        "plain_res64": (W.plain_cloud(300, 21), 64),
        "clusters_res512": (W.cluster_cloud(300, 22, clusters=4), 512),
        "pytest32_res4096": (W.pytest_cloud(), 4096),
        "faint_res256": (faint, 256),
    }


def voxelbvh_fixture(L, cloud, res, T=None):
    n = cloud.n
    m, q, s, o = (_f(cloud[k]) for k in ("means", "quats", "scales", "opacities"))
    Ti = None if T is None else np.linalg.inv(T.astype(np.float64)).astype(np.float32)
    box = O.voxelbvh_ijkl(cloud, res, T, Ti)["world_bbox"]  # a min / max over the Gaussians' boxes
    pad = 8 * 256 * ((n + 255) // 256)
    k = np.zeros(pad, np.uint64)
    i = np.zeros(pad, np.uint32)
    Tp = None if T is None else _f(T).reshape(16)
    Tip = None if Ti is None else _f(Ti).reshape(16)
    L.ref_voxelbvh_to_ijkl(n, res, m.ctypes.data, o.ctypes.data, q.ctypes.data, s.ctypes.data,
                           None if Tp is None else Tp.ctypes.data, None if Tip is None else Tip.ctypes.data,
                           _f(box).ctypes.data, k.ctypes.data, i.ctypes.data)
    k, i = k[: 8 * n], i[: 8 * n]
    order = np.argsort(k, kind="stable")
    k, i = np.ascontiguousarray(k[order]), np.ascontiguousarray(i[order])
    N = k.size
    starts, scan = np.zeros(N, np.uint32), np.zeros(N, np.uint32)
    headers = np.zeros(2 * N, np.uint32)
    L.ref_voxelbvh_ranges(N, k.ctypes.data, starts.ctypes.data, scan.ctypes.data, headers.ctypes.data)
    extra = {} if T is None else {"transform": _f(T), "transform_inv": _f(Ti)}
    return dict(means=m, quats=q, scales=s, opacities=o, resolution=np.uint32(res), world_bbox=_f(box),
                ijkl=k, prim_id=i, range=headers, ranges=np.int64(scan[-1] if N else 0), **extra)


def load_ref_topology():
    L = load_ref()
    L.ref_node2_build.restype = ctypes.c_int64
    L.ref_node2_build.argtypes = [ctypes.c_int64] + [P] * 4 + [ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32, P, P]
    L.ref_node2_copy.restype = ctypes.c_int64
    L.ref_node2_copy.argtypes = [P, ctypes.c_int64]
    return L


# the reference's batch sizes (raster/Raster.cpp:443-444)
PRIM_BATCH = 256 * 1024
IJK_BATCH = 8 * 1024 * 1024


def inputs_sha256(cloud) -> str:
    h = hashlib.sha256()
    for k in ("means", "quats", "scales", "opacities"):
        h.update(_f(cloud[k]).tobytes())
    return h.hexdigest()


def topology_fixture(L, cloud, vs, keep_bytes):
    m, q, s, o = (_f(cloud[k]) for k in ("means", "quats", "scales", "opacities"))
    cnt = np.zeros(5, np.int64)
    bb = np.zeros(6, np.int32)
    nb = L.ref_node2_build(cloud.n, m.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, vs, PRIM_BATCH,
                           IJK_BATCH, cnt.ctypes.data, bb.ctypes.data)
    if nb <= 0:
        raise SystemExit("reference grid build failed")
    region = np.empty(nb, np.uint8)
    L.ref_node2_copy(region.ctypes.data, nb)
    out = dict(voxel_size=np.float32(vs), node2_sha256=np.array(hashlib.sha256(region.tobytes()).hexdigest()),
               node2_bytes=np.int64(nb), upper=np.int64(cnt[0]), lower=np.int64(cnt[1]), leaf=np.int64(cnt[2]),
               value_count=np.int64(cnt[3]), windows=np.int64(cnt[4]), bbox=bb)
    if keep_bytes:
        out["node2"] = region
    return out


def topology_cases():
    """(cloud, voxel size, regeneration spec or None, keep the region bytes)"""
    cases = {name: (c, vs, None, name in ("tiny", "pytest32", "plain", "aniso")) for name, (c, vs) in raster_cases().items()}
    cases["windows_100k"] = (W.plain_cloud(100_000, 0), 0.01, ("plain_cloud", 100_000, 0), False)
    cases["batches_300k"] = (W.plain_cloud(300_000, 0), 0.04, ("plain_cloud", 300_000, 0), False)
    return cases


def write_topology(L):
    for name, (cloud, vs, spec, keep) in topology_cases().items():
        z = topology_fixture(L, cloud, vs, keep)
        if spec is None:
            z.update(means=_f(cloud["means"]), quats=_f(cloud["quats"]), scales=_f(cloud["scales"]),
                     opacities=_f(cloud["opacities"]))
        else:
            z.update(generator=np.array(spec[0]), count=np.int64(spec[1]), seed=np.int64(spec[2]),
                     inputs_sha256=np.array(inputs_sha256(cloud)))
        np.savez_compressed(os.path.join(HERE, f"topology_{name}.npz"), **z)
        print("topology", name, int(z["windows"]), "windows", str(z["node2_sha256"])[:16])


def main():
    if "--topology" in sys.argv:
        write_topology(load_ref_topology())
        return
    L = load_ref()
    for name, (cloud, vs) in raster_cases().items():
        np.savez_compressed(os.path.join(HERE, f"raster_{name}.npz"), **raster_fixture(L, cloud, vs))
    # a tighter cull radius (gaussian_frag_color.slang:205, the shader parameter)
    cloud, vs = raster_cases()["clusters"]
    np.savez_compressed(os.path.join(HERE, "raster_clusters_cull0.01.npz"), **raster_fixture(L, cloud, vs, cull=0.01))
    for name, (cloud, res) in voxelbvh_cases().items():
        np.savez_compressed(os.path.join(HERE, f"voxelbvh_{name}.npz"), **voxelbvh_fixture(L, cloud, res))
    # a transform (rows of the reference's pnanovdb_camera_mat_t, row vectors):
    # rotation about z, uniform scale 1.5, translation
    ang = 0.7
    T = np.eye(4)
    T[:3, :3] = np.array([[np.cos(ang), np.sin(ang), 0], [-np.sin(ang), np.cos(ang), 0], [0, 0, 1]]) * 1.5
    T[3, :3] = [0.3, -2.0, 5.0]
    cloud, res = voxelbvh_cases()["clusters_res512"]
    np.savez_compressed(os.path.join(HERE, "voxelbvh_clusters_res512_transform.npz"),
                        **voxelbvh_fixture(L, cloud, res, T.astype(np.float32)))
    write_topology(load_ref_topology())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
