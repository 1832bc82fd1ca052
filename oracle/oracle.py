"""ctypes wrapper of the CPU oracle (oracle/_build/libvox_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker; never by the product.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_float, c_int, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libvox_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_shaders.so")

OV_MODE_WINDOWS = 1
OV_MODE_NO_F64 = 2
OV_MODE_SMOOTH = 4

COUNT_NAMES = ["G", "G_valid", "F", "P", "V", "upper", "lower", "leaf", "value_count", "node2_bytes", "windows", "error"]


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    else:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def build_ref() -> str | None:
    """Compiles the reference's shaders as C++ when the reference checkout exists."""
    script = os.path.join(HERE, "ref_shaders", "build_ref.sh")
    subprocess.run(["sh", script], check=True, stdout=subprocess.DEVNULL)
    return REF_PATH if os.path.exists(REF_PATH) else None


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.ov_run.restype = c_void_p
        L.ov_run.argtypes = [c_int64] + [c_void_p] * 5 + [c_float, c_float, c_int, c_int]
        L.ov_destroy.argtypes = [c_void_p]
        L.ov_counts.argtypes = [c_void_p, c_void_p]
        L.ov_chan_math.argtypes = [c_int64] + [c_void_p] * 6
        L.ov_chan_math.restype = None
        L.ov_node2_bytes.restype = c_int64
        L.ov_node2_bytes.argtypes = [c_void_p, c_void_p]
        L.ov_pairs.argtypes = [c_void_p, c_void_p, c_void_p]
        L.ov_values.argtypes = [c_void_p] + [c_void_p] * 5
        L.ov_voxels.argtypes = [c_void_p, c_void_p, c_void_p]
        L.ov_bbox.argtypes = [c_void_p, c_void_p]
        L.ov_node_table.argtypes = [c_void_p] + [c_void_p] * 4
        L.ov_preprocess.argtypes = [c_int64] + [c_void_p] * 8
        L.ov_prim_bbox.restype = c_int
        L.ov_prim_bbox.argtypes = [c_void_p, c_void_p, c_void_p, c_float, c_float, c_void_p, c_void_p]
        L.ov_frag_test.restype = c_int
        L.ov_frag_test.argtypes = [c_void_p, c_void_p, c_void_p, c_float, c_float, c_void_p, c_void_p, c_void_p]
        L.ov_frag_rgba.restype = ctypes.c_uint32
        L.ov_frag_rgba.argtypes = [c_void_p, c_void_p, c_void_p, c_float, c_void_p, c_float, c_float, c_void_p, c_void_p]
        L.ov_hier_key.restype = ctypes.c_uint64
        L.ov_hier_key.argtypes = [ctypes.c_int32] * 3
        L.ov_lookup.restype = c_int64
        L.ov_lookup.argtypes = [c_void_p] + [ctypes.c_int32] * 3
        L.ov_smooth_grad64.restype = c_int
        L.ov_smooth_grad64.argtypes = [c_void_p] + [c_void_p] * 5 + [c_int] + [c_void_p] * 7
        L.ov_smooth_loss64.restype = ctypes.c_double
        L.ov_smooth_loss64.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p]
        L.ov_voxelbvh_ijkl.argtypes = [c_int64] + [c_void_p] * 4 + [ctypes.c_uint32] + [c_void_p] * 6 + [c_int]
        L.ov_voxelbvh_ijkl.restype = c_int64
        _LIB = L
    return _LIB


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def preprocess(raw):
    """A2 restatement: raw [means, logit, quats, log scales, sh0, sh_n] -> activated dict."""
    means, logit, quats, log_s, sh0 = (_f32(raw[i]) for i in range(5))
    n = means.reshape(-1, 3).shape[0]
    q = np.empty((n, 4), np.float32)
    s = np.empty((n, 3), np.float32)
    o = np.empty(n, np.float32)
    c = np.empty((n, 3), np.float32)
    lib().ov_preprocess(n, quats.ctypes.data, log_s.ctypes.data, logit.ctypes.data, sh0.ctypes.data, q.ctypes.data, s.ctypes.data, o.ctypes.data, c.ctypes.data)
    return {"means": means.reshape(n, 3), "quats": q, "scales": s, "opacities": o, "colors": c}


class OracleResult:
    def __init__(self, cloud, voxel_size, cull_scale=0.0, window_mode=0, nthreads=None):
        L = lib()
        self._keep = [_f32(cloud[k]) for k in ("means", "quats", "scales", "colors", "opacities")]
        n = self._keep[0].reshape(-1, 3).shape[0]
        nthreads = nthreads or max(1, min(16, os.cpu_count() or 1))
        self.h = L.ov_run(n, *[a.ctypes.data for a in self._keep], float(voxel_size), float(cull_scale), int(window_mode), int(nthreads))
        cnt = np.zeros(12, np.int64)
        L.ov_counts(self.h, cnt.ctypes.data)
        self.counts = dict(zip(COUNT_NAMES, cnt.tolist()))

    def close(self):
        if self.h:
            lib().ov_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def node2(self) -> np.ndarray:
        out = np.empty(self.counts["node2_bytes"], np.uint8)
        lib().ov_node2_bytes(self.h, out.ctypes.data)
        return out

    def pairs(self):
        P = self.counts["P"]
        k = np.empty(P, np.uint64)
        i = np.empty(P, np.uint32)
        lib().ov_pairs(self.h, k.ctypes.data, i.ctypes.data)
        return k, i

    def values(self):
        vc = self.counts["value_count"]
        rgba = np.empty(vc, np.uint32)
        d = np.empty(vc, np.float32)
        c = np.empty((vc, 3), np.float32)
        d64 = np.empty(vc, np.float64)
        c64 = np.empty((vc, 3), np.float64)
        lib().ov_values(self.h, rgba.ctypes.data, d.ctypes.data, c.ctypes.data, d64.ctypes.data, c64.ctypes.data)
        return {"rgba8": rgba, "density": d, "color": c, "density64": d64, "color64": c64}

    def voxels(self):
        V = self.counts["V"]
        ijk = np.empty((V, 3), np.int32)
        vidx = np.empty(V, np.uint64)
        lib().ov_voxels(self.h, ijk.ctypes.data, vidx.ctypes.data)
        return ijk, vidx

    def bbox(self):
        b = np.empty(6, np.int32)
        lib().ov_bbox(self.h, b.ctypes.data)
        return b

    def lookup(self, i, j, k) -> int:
        return int(lib().ov_lookup(self.h, int(i), int(j), int(k)))

    def smooth_grad64(self, params, raw, grad_density, grad_color=None):
        """FP64 adjoint of the smooth channels.  params: dict means/quats/scales/
        opacities/colors as passed to the product (raw: quats before normalisation,
        log-scales, opacity logits, SH0).  grad arrays are indexed by value index."""
        arrs = [_f32(params[k]) for k in ("means", "quats", "scales", "opacities", "colors")]
        n = arrs[0].reshape(-1, 3).shape[0]
        gd = np.ascontiguousarray(grad_density, np.float64)
        gc = None if grad_color is None else np.ascontiguousarray(grad_color, np.float64)
        out = {
            "means": np.zeros((n, 3)),
            "quats": np.zeros((n, 4)),
            "scales": np.zeros((n, 3)),
            "opacities": np.zeros(n),
            "colors": np.zeros((n, 3)),
        }
        rc = lib().ov_smooth_grad64(
            self.h, *[a.ctypes.data for a in arrs], int(bool(raw)), gd.ctypes.data, None if gc is None else gc.ctypes.data,
            *[out[k].ctypes.data for k in ("means", "quats", "scales", "opacities", "colors")])
        if rc != 0:
            raise RuntimeError("oracle adjoint failed")
        return out

    def smooth_loss64(self, theta, raw, grad_density, grad_color=None):
        """FP64 contribution of one Gaussian theta = [mean3, quat wxyz4, scale3, opacity, colour3]."""
        t = np.ascontiguousarray(theta, np.float64)
        gd = np.ascontiguousarray(grad_density, np.float64)
        gc = None if grad_color is None else np.ascontiguousarray(grad_color, np.float64)
        return float(lib().ov_smooth_loss64(self.h, t.ctypes.data, int(bool(raw)), gd.ctypes.data,
                                            None if gc is None else gc.ctypes.data))


def hier_key(i, j, k) -> int:
    return int(lib().ov_hier_key(int(i), int(j), int(k)))


def voxelbvh_ijkl(cloud, resolution: int, transform=None, transform_inv=None, nthreads=None):
    """VoxelBVH Gaussian ingestion (raster/VoxelBVH.cpp:1225-1435) of an
    activated cloud: sorted 64-bit cell keys, their Gaussian ids, the
    [start, end) header of every distinct key (zeros past `ranges`) and the
    world box.  transform / transform_inv: 4x4 float32 (row-vector
    convention, p' = [p 1] T) or None for the identity."""
    means, q, s, o = (_f32(cloud[k]) for k in ("means", "quats", "scales", "opacities"))
    n = means.reshape(-1, 3).shape[0]
    T = None if transform is None else _f32(transform).reshape(16)
    Ti = None if transform_inv is None else _f32(transform_inv).reshape(16)
    keys = np.empty(8 * n, np.uint64)
    ids = np.empty(8 * n, np.uint32)
    rng = np.empty(16 * n, np.uint32)
    box = np.empty(6, np.float32)
    r = lib().ov_voxelbvh_ijkl(n, means.ctypes.data, o.ctypes.data, q.ctypes.data, s.ctypes.data, int(resolution),
                               None if T is None else T.ctypes.data, None if Ti is None else Ti.ctypes.data,
                               keys.ctypes.data, ids.ctypes.data, rng.ctypes.data, box.ctypes.data,
                               int(nthreads or max(1, min(16, os.cpu_count() or 1))))
    return {"ijkl": keys, "prim_id": ids, "range": rng, "ranges": int(r), "world_bbox": box}


def chan_math(x, b, e):
    """The float channels' exp(x), log(b), b^e (float32 arrays of one length)."""
    x, b, e = (np.ascontiguousarray(a, dtype=np.float32) for a in (x, b, e))
    n = x.shape[0]
    out = [np.empty(n, np.float32) for _ in range(3)]
    lib().ov_chan_math(n, x.ctypes.data, b.ctypes.data, e.ctypes.data, *(o.ctypes.data for o in out))
    return out
