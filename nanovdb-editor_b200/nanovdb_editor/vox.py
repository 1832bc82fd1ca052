"""Low-level binding of the library's vox_* entry points (include/pnanovdb_b200.h).

``VoxContext.voxelize`` takes CUDA tensors (device pointers, no copies) and
returns the grid as a ``NodeGrid`` on the host or leaves it on the device;
``voxelize_host`` takes numpy arrays and times host<->device copies inside
the call (the end-to-end path of ``raster_to_nanovdb``).
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, Structure, byref, c_char_p, c_float, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p

import numpy as np

from .exceptions import PipelineError
from .grid import NodeGrid
from .utils import load_library

FLAG_RAW_INPUTS = 1
FLAG_WINDOW_ORDER = 2
FLAG_DIFFERENTIABLE = 4
FLAG_BF16_INPUTS = 8

STATUS = {
    0: "ok",
    -1: "invalid arguments",
    -2: "CUDA error",
    -3: "out of device memory",
    -4: "voxel coordinate outside [-65536, 65535]",
    -5: "Gaussian bbox covers 2^31 or more voxels",
    -6: "bounded device wait expired",
    -7: "buffer too small",
}


class vox_gaussians_t(Structure):
    _fields_ = [
        ("means", c_void_p),
        ("quats", c_void_p),
        ("scales", c_void_p),
        ("opacities", c_void_p),
        ("colors", c_void_p),
        ("count", c_int64),
    ]


class vox_stats_t(Structure):
    _fields_ = [
        ("gaussians", c_int64),
        ("candidates", c_int64),
        ("pairs", c_int64),
        ("voxels", c_int64),
        ("uppers", c_int64),
        ("lowers", c_int64),
        ("leaves", c_int64),
        ("value_count", c_int64),
        ("grid_bytes", c_int64),
        ("key_bits", c_int32),
        ("sort_passes", c_int32),
        ("ms_prep", c_float),
        ("ms_emit", c_float),
        ("ms_sort", c_float),
        ("ms_build", c_float),
        ("ms_accumulate", c_float),
        ("ms_total", c_float),
        ("kernel_launches", c_int64),
        ("ms_backward", c_float),
        ("sort_shape", c_int32),
        ("leaf_pairs", c_int64),
        ("candidate_leaves", c_int64),
        ("ms_vb_keys", c_float),
        ("ms_vb_sort", c_float),
        ("ms_vb_ranges", c_float),
        ("vb_sort_bits", c_int32),
        ("vb_launches", c_int64),
        ("walk_ctas_per_sm", c_int32),
        ("vb_search", c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _lib():
    lib = load_library("pnanovdbcompute")
    if not getattr(lib, "_vox_bound", False):
        lib.vox_context_create.restype = c_void_p
        lib.vox_context_create.argtypes = [c_int]
        lib.vox_context_destroy.argtypes = [c_void_p]
        lib.vox_context_stream.restype = c_void_p
        lib.vox_context_stream.argtypes = [c_void_p]
        lib.vox_last_error.restype = c_char_p
        lib.vox_last_error.argtypes = [c_void_p]
        lib.vox_voxelize.restype = c_int
        lib.vox_voxelize.argtypes = [c_void_p, POINTER(vox_gaussians_t), c_float, c_float, c_uint32, POINTER(c_void_p), POINTER(c_uint64)]
        lib.vox_voxelize_host.restype = c_int
        lib.vox_voxelize_host.argtypes = [c_void_p, POINTER(vox_gaussians_t), c_float, c_float, c_uint32, c_void_p, c_uint64, POINTER(c_uint64)]
        lib.vox_copy_grid.restype = c_int
        lib.vox_copy_grid.argtypes = [c_void_p, c_void_p, c_uint64]
        lib.vox_copy_pairs.restype = c_int
        lib.vox_copy_pairs.argtypes = [c_void_p, c_void_p, c_void_p, c_int64]
        lib.vox_get_stats.argtypes = [c_void_p, POINTER(vox_stats_t)]
        lib.vox_global_scan_u64.restype = c_int
        lib.vox_global_scan_u64.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p]
        lib.vox_voxelize_batch.restype = c_int
        lib.vox_voxelize_batch.argtypes = [c_void_p, POINTER(vox_gaussians_t), c_int64, c_void_p, c_void_p, c_float, c_uint32, POINTER(c_void_p), c_void_p, c_void_p]
        lib.vox_voxel_coords.restype = c_int
        lib.vox_voxel_coords.argtypes = [c_void_p, c_void_p, c_int64]
        lib.vox_backward.restype = c_int
        lib.vox_backward.argtypes = [c_void_p, POINTER(vox_gaussians_t)] + [c_void_p] * 7
        lib.vox_radix_sort_key64.restype = c_int
        lib.vox_radix_sort_key64.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_uint32]
        lib.vox_global_scan_u32.restype = c_int
        lib.vox_global_scan_u32.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_int, c_void_p]
        lib.vox_global_scan_max_u32.restype = c_int
        lib.vox_global_scan_max_u32.argtypes = [c_void_p, c_void_p, c_void_p, c_int64]
        lib.vox_radix_sort_u32.restype = c_int
        lib.vox_radix_sort_u32.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_uint32]
        lib.vox_radix_sort_dual_key.restype = c_int
        lib.vox_radix_sort_dual_key.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_uint32, c_uint32]
        lib.vox_voxelbvh_ijkl_from_gaussians.restype = c_int
        lib.vox_voxelbvh_ijkl_from_gaussians.argtypes = [c_void_p] + [c_void_p] * 4 + [c_int64, c_uint32] + [c_void_p] * 5 + [POINTER(c_int64)]
        lib.vox_voxelbvh_ijkl_from_gaussians_file.restype = c_int
        lib.vox_voxelbvh_ijkl_from_gaussians_file.argtypes = [c_void_p, ctypes.c_char_p, c_uint32, c_void_p] + [c_void_p] * 5 + [c_uint32]
        lib.vox_voxelbvh_transform_inverse.restype = c_int
        lib.vox_voxelbvh_transform_inverse.argtypes = [c_void_p, c_void_p]
        lib.vox_context_set_wait_limit.restype = c_int
        lib.vox_context_set_wait_limit.argtypes = [c_void_p, c_uint32, c_int]
        lib.vox_adam_bf16.restype = c_int
        lib.vox_adam_bf16.argtypes = [c_void_p] * 5 + [c_int64, c_float, c_float, c_float, c_float, c_int64, c_void_p]
        lib._vox_bound = True
    return lib


def _ptr(t) -> int:
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return int(t.data_ptr())
    return int(t.ctypes.data)


class VoxContext:
    """One CUDA stream + persistent device buffers on one device."""

    def __init__(self, device: int = 0):
        self.lib = _lib()
        self.handle = self.lib.vox_context_create(int(device))
        if not self.handle:
            raise PipelineError("vox_context_create failed (no CUDA device?)")
        self.last_grid_bytes = 0
        self.generation = 0  # counts forward calls; the adjoint belongs to the latest

    def close(self):
        if getattr(self, "handle", None):
            self.lib.vox_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self.lib.vox_context_stream(self.handle) or 0)

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.vox_last_error(self.handle).decode(errors="replace")
            raise PipelineError(f"{what}: {STATUS.get(rc, rc)}: {msg}")

    @staticmethod
    def _gauss(means, quats, scales, opacities, colors) -> vox_gaussians_t:
        n = int(means.shape[0]) if len(means.shape) > 1 else int(means.shape[0]) // 3
        g = vox_gaussians_t()
        g.means, g.quats, g.scales, g.opacities, g.colors = (
            _ptr(means),
            _ptr(quats),
            _ptr(scales),
            _ptr(opacities),
            _ptr(colors),
        )
        g.count = n
        return g

    def voxelize(self, means, quats, scales, opacities, colors, voxel_size, cull_scale=0.05, flags=0):
        """Device tensors in (contiguous float32 CUDA tensors); returns (device ptr, bytes).

        The caller must have finished producing the inputs (e.g. torch.cuda.synchronize()).
        """
        g = self._gauss(means, quats, scales, opacities, colors)
        ptr = c_void_p()
        nbytes = c_uint64()
        self.generation += 1
        rc = self.lib.vox_voxelize(self.handle, byref(g), float(voxel_size), float(cull_scale), int(flags), byref(ptr), byref(nbytes))
        self._check(rc, "vox_voxelize")
        self.last_grid_bytes = int(nbytes.value)
        return int(ptr.value or 0), int(nbytes.value)

    def voxelize_batch(self, means, quats, scales, opacities, colors, cloud_start, voxel_sizes, cull_scale=0.05, flags=0):
        """Many clouds in one call (device tensors, concatenated).  cloud_start: host
        int64 [B + 1]; voxel_sizes: host float32 [B].  Returns (device ptr, grid
        offsets [B + 1], value offsets [B + 1]) - grid b is bytes [off[b], off[b + 1])."""
        g = self._gauss(means, quats, scales, opacities, colors)
        cs = np.ascontiguousarray(cloud_start, dtype=np.int64)
        vs = np.ascontiguousarray(voxel_sizes, dtype=np.float32)
        B = int(vs.shape[0])
        if cs.shape[0] != B + 1:
            raise PipelineError("voxelize_batch: cloud_start needs one more entry than voxel_sizes")
        goff = np.zeros(B + 1, dtype=np.uint64)
        voff = np.zeros(B + 1, dtype=np.uint64)
        ptr = c_void_p()
        self.generation += 1
        rc = self.lib.vox_voxelize_batch(self.handle, byref(g), B, cs.ctypes.data, vs.ctypes.data, float(cull_scale), int(flags),
                                         byref(ptr), goff.ctypes.data, voff.ctypes.data)
        self._check(rc, "vox_voxelize_batch")
        self.last_grid_bytes = int(goff[-1])
        return int(ptr.value or 0), goff, voff

    def grids(self, grid_offsets) -> list:
        """Host copies of every cloud's grid of the last batched call."""
        buf = np.empty(self.last_grid_bytes, dtype=np.uint8)
        self._check(self.lib.vox_copy_grid(self.handle, buf.ctypes.data, buf.nbytes), "vox_copy_grid")
        return [NodeGrid(buf[int(a) : int(b)]) for a, b in zip(grid_offsets[:-1], grid_offsets[1:])]

    def voxelize_host(self, means, quats, scales, opacities, colors, voxel_size, cull_scale=0.05, flags=0) -> NodeGrid:
        """numpy float32 arrays in, host grid out (copies counted in the call)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (means, quats, scales, opacities, colors)]
        g = self._gauss(*arrs)
        nbytes = c_uint64()
        self.generation += 1
        rc = self.lib.vox_voxelize_host(self.handle, byref(g), float(voxel_size), float(cull_scale), int(flags), None, 0, byref(nbytes))
        self._check(rc, "vox_voxelize_host")
        self.last_grid_bytes = int(nbytes.value)
        return self.grid()

    def backward(self, means, quats, scales, opacities, colors, grad_density, grad_color, out):
        """Adjoint of the last differentiable voxelize (device tensors).  `out` maps
        means/quats/scales/opacities/colors to float32 CUDA tensors (or None)."""
        g = self._gauss(means, quats, scales, opacities, colors)
        rc = self.lib.vox_backward(
            self.handle, byref(g), _ptr(grad_density), _ptr(grad_color),
            *[_ptr(out.get(k)) for k in ("means", "quats", "scales", "opacities", "colors")])
        self._check(rc, "vox_backward")

    def voxel_coords(self, dst) -> None:
        """Writes the active voxels' (i, j, k) into a CUDA int32 tensor [value_count, 3], row = value index
        (background rows untouched)."""
        self._check(self.lib.vox_voxel_coords(self.handle, _ptr(dst), int(dst.shape[0]) if dst.dim() > 1 else int(dst.numel()) // 3), "vox_voxel_coords")

    def grid_device(self, dst) -> None:
        """Copies the last grid into a CUDA uint8 tensor of at least last_grid_bytes."""
        self._check(self.lib.vox_copy_grid(self.handle, _ptr(dst), int(dst.numel())), "vox_copy_grid")

    def grid(self) -> NodeGrid:
        out = np.empty(self.last_grid_bytes, dtype=np.uint8)
        self._check(self.lib.vox_copy_grid(self.handle, out.ctypes.data, out.nbytes), "vox_copy_grid")
        return NodeGrid(out)

    def pairs(self):
        st = self.stats()
        n = int(st["pairs"])
        keys = np.empty(n, dtype=np.uint64)
        ids = np.empty(n, dtype=np.uint32)
        self._check(self.lib.vox_copy_pairs(self.handle, keys.ctypes.data, ids.ctypes.data, n), "vox_copy_pairs")
        return keys, ids

    def stats(self) -> dict:
        st = vox_stats_t()
        self.lib.vox_get_stats(self.handle, byref(st))
        return st.as_dict()

    def adam_bf16(self, master, m, v, grad, out_bf16, step: int, lr: float, beta1: float = 0.9, beta2: float = 0.999,
                  eps: float = 1e-8) -> None:
        """One fused Adam step on the context's stream: FP32 master / moments
        (float32 CUDA tensors) updated from `grad`, the bfloat16 attribute
        tensor `out_bf16` rewritten from the master copy."""
        n = int(master.numel())
        for t in (m, v, grad, out_bf16):
            if int(t.numel()) != n:
                raise PipelineError("adam_bf16: tensors of different sizes")
        rc = self.lib.vox_adam_bf16(_ptr(master), _ptr(m), _ptr(v), _ptr(grad), _ptr(out_bf16), n, float(lr), float(beta1),
                                    float(beta2), float(eps), int(step), self.stream)
        if rc != 0:
            raise PipelineError(f"vox_adam_bf16: {STATUS.get(rc, rc)}")

    def set_wait_limit(self, max_polls=None, withhold_publication: bool = False) -> None:
        """Bound of the device look-back waits for later calls (None: the
        default); withhold_publication makes every wait run out (a test of the
        VOX_ERR_TIMEOUT path)."""
        polls = 0xFFFFFFFF if max_polls is None else int(max_polls)
        self._check(self.lib.vox_context_set_wait_limit(self.handle, polls, 1 if withhold_publication else 0), "set_wait_limit")

    def global_scan_u64(self, d_in, d_out, d_total, inclusive: bool = True) -> None:
        """Scan of CUDA uint64 tensors (the reference's global_scan_uint64 is inclusive)."""
        n = int(d_in.numel())
        self._check(self.lib.vox_global_scan_u64(self.handle, _ptr(d_in), _ptr(d_out), n, 1 if inclusive else 0, _ptr(d_total)), "vox_global_scan_u64")

    def voxelbvh_ijkl_from_gaussians(self, means, opacities, quats, scales, resolution: int, transform=None):
        """VoxelBVH Gaussian ingestion (the reference's ijkl_from_gaussians,
        raster/VoxelBVH.cpp:1225-1435) of activated CUDA float32 tensors
        (quaternions w x y z).  Returns a dict of CUDA tensors: ``ijkl``
        (int64 holding the uint64 keys, 8 per Gaussian, sorted), ``prim_id``
        (int32 holding uint32 ids), ``range`` (int32 holding uint32
        [start, end) pairs, 16 per Gaussian), ``world_bbox`` (6 floats) and the
        int ``range_count``.  ``transform``: 4x4 (row-vector convention,
        p' = [p 1] M) or None."""
        import torch

        n = int(means.shape[0]) if means.dim() > 0 else 0
        dev = means.device
        ijkl = torch.empty(8 * n, dtype=torch.int64, device=dev)
        prim_id = torch.empty(8 * n, dtype=torch.int32, device=dev)
        rng = torch.empty(16 * n, dtype=torch.int32, device=dev)
        box = torch.empty(6, dtype=torch.float32, device=dev)
        T = None
        if transform is not None:
            T = np.ascontiguousarray(np.asarray(transform, dtype=np.float32).reshape(16))
        count = c_int64(0)
        args = [means.contiguous(), opacities.contiguous(), quats.contiguous(), scales.contiguous()]
        for a in args:
            if a.dtype != torch.float32 or a.device != dev:
                raise ValueError("voxelbvh_ijkl_from_gaussians takes float32 tensors on one device")
        # the library works on its own stream: let torch's finish producing the
        # inputs and releasing the outputs' memory first
        torch.cuda.current_stream(dev).synchronize()
        self._check(self.lib.vox_voxelbvh_ijkl_from_gaussians(self.handle, *[_ptr(a) for a in args], n, int(resolution),
                                                              _ptr(T), _ptr(ijkl), _ptr(prim_id), _ptr(rng), _ptr(box),
                                                              byref(count)), "vox_voxelbvh_ijkl_from_gaussians")
        return {"ijkl": ijkl, "prim_id": prim_id, "range": rng, "world_bbox": box, "range_count": int(count.value)}

    def voxelbvh_ijkl_from_file(self, filename: str, resolution: int, transform=None) -> dict:
        """VoxelBVH ingestion of a Gaussian file (the reference's
        ijkl_from_gaussians_file, raster/VoxelBVH.cpp:1437-1575): .npz or .ply
        with raw attributes, activated on the host.  Returns numpy arrays
        ``ijkl`` (uint64), ``prim_id`` (uint32), ``range`` (uint32 pairs),
        ``world_bbox`` and the activated ``means``, ``opacities``,
        ``quaternions``, ``scales``."""
        from .compute import Compute, pnanovdb_ComputeArray

        T = None
        if transform is not None:
            T = np.ascontiguousarray(np.asarray(transform, dtype=np.float32).reshape(16))
        outs = [POINTER(pnanovdb_ComputeArray)() for _ in range(4)]
        garr = (POINTER(pnanovdb_ComputeArray) * 6)()
        self._check(self.lib.vox_voxelbvh_ijkl_from_gaussians_file(
            self.handle, str(filename).encode(), int(resolution), _ptr(T), *[ctypes.addressof(o) for o in outs],
            ctypes.addressof(garr), 6), "vox_voxelbvh_ijkl_from_gaussians_file")
        comp = Compute()

        def take(ptr, dtype):
            a = ptr.contents
            nbytes = int(a.element_size * a.element_count)
            out = np.frombuffer((ctypes.c_byte * nbytes).from_address(a.data), dtype=dtype).copy() if nbytes else np.zeros(0, dtype)
            comp.destroy_array(a)
            return out

        res = {"ijkl": take(outs[0], np.uint64), "prim_id": take(outs[1], np.uint32),
               "range": take(outs[2], np.uint32), "world_bbox": take(outs[3], np.float32)}
        for name, ptr in zip(("means", "opacities", "quaternions", "scales", "sh_0", "sh_n"), garr):
            res[name] = take(ptr, np.float32)
        return res

    def voxelbvh_transform_inverse(self, transform):
        """The float32 inverse vox_voxelbvh_ijkl_from_gaussians applies for `transform` (4x4)."""
        m = np.ascontiguousarray(np.asarray(transform, dtype=np.float32).reshape(16))
        out = np.empty(16, np.float32)
        self._check(self.lib.vox_voxelbvh_transform_inverse(m.ctypes.data, out.ctypes.data), "vox_voxelbvh_transform_inverse")
        return out.reshape(4, 4)

    def global_scan_u32(self, d_in, d_out, d_total=None, inclusive: bool = True) -> None:
        """Scan of CUDA uint32 tensors (int32 storage), sums mod 2^32 (the reference's global_scan)."""
        n = int(d_in.numel())
        self._check(self.lib.vox_global_scan_u32(self.handle, _ptr(d_in), _ptr(d_out), n, 1 if inclusive else 0, _ptr(d_total)), "vox_global_scan_u32")

    def global_scan_max_u32(self, d_in, d_out) -> None:
        """Inclusive running maximum of CUDA uint32 tensors (the reference's global_scan_max)."""
        n = int(d_in.numel())
        self._check(self.lib.vox_global_scan_max_u32(self.handle, _ptr(d_in), _ptr(d_out), n), "vox_global_scan_max_u32")

    def radix_sort_u32(self, d_keys, d_vals, key_bits: int = 32) -> None:
        """Stable in-place sort of CUDA (uint32 key, uint32 value) tensors by key bits [0, key_bits)."""
        n = int(d_keys.numel())
        self._check(self.lib.vox_radix_sort_u32(self.handle, _ptr(d_keys), _ptr(d_vals), n, int(key_bits)), "vox_radix_sort_u32")

    def radix_sort_dual_key(self, d_low, d_high, d_vals, low_bits: int = 32, high_bits: int = 32) -> None:
        """Stable in-place sort of CUDA uint32 (low key, high key, value) tensors by (high, low)."""
        n = int(d_low.numel())
        self._check(self.lib.vox_radix_sort_dual_key(self.handle, _ptr(d_low), _ptr(d_high), _ptr(d_vals), n, int(low_bits), int(high_bits)), "vox_radix_sort_dual_key")

    def radix_sort_key64(self, d_keys, d_vals, key_bits: int = 64) -> None:
        """Stable in-place sort of CUDA (uint64 key, uint32 value) tensors by key bits [0, key_bits)."""
        n = int(d_keys.numel())
        self._check(self.lib.vox_radix_sort_key64(self.handle, _ptr(d_keys), _ptr(d_vals), n, int(key_bits)), "vox_radix_sort_key64")
