"""ctypes mirror of ``pnanovdb_raster_t`` (pymodule/nanovdb_editor/raster.py:14-279).

Same structure layout, method names, argument meaning and error behaviour as
the reference binding; the table comes from this library's
``pnanovdb_get_raster()``.
"""

from __future__ import annotations

from ctypes import CFUNCTYPE, POINTER, Structure, byref, c_char_p, c_float, c_int32, c_uint32, c_uint64, c_void_p, pointer

from .compute import Compute, pnanovdb_Compute, pnanovdb_ComputeArray
from .exceptions import InvalidArgumentError
from .utils import load_library

COMPUTE_LIB = "pnanovdbcompute"


class pnanovdb_Raster(Structure):
    """Definition equivalent to pnanovdb_raster_t (Raster.h:58-174)."""

    _fields_ = [
        ("interface_pnanovdb_reflect_data_type", c_void_p),
        ("compute", POINTER(pnanovdb_Compute)),
        ("create_context", CFUNCTYPE(c_void_p, POINTER(pnanovdb_Compute), c_void_p)),
        ("destroy_context", CFUNCTYPE(None, POINTER(pnanovdb_Compute), c_void_p, c_void_p)),
        (
            "create_gaussian_data",
            CFUNCTYPE(
                c_void_p,
                POINTER(pnanovdb_Compute),
                c_void_p,
                c_void_p,
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(POINTER(pnanovdb_ComputeArray)),
                c_void_p,
            ),
        ),
        ("upload_gaussian_data", CFUNCTYPE(None, POINTER(pnanovdb_Compute), c_void_p, c_void_p, c_void_p)),
        ("destroy_gaussian_data", CFUNCTYPE(None, POINTER(pnanovdb_Compute), c_void_p, c_void_p)),
        (
            "raster_gaussian_2d",
            CFUNCTYPE(
                None,
                POINTER(pnanovdb_Compute),
                c_void_p,
                c_void_p,
                c_void_p,
                c_void_p,
                c_uint32,
                c_uint32,
                c_void_p,
                c_void_p,
                c_void_p,
                c_uint32,
            ),
        ),
        (
            "raster_gaussian_3d",
            CFUNCTYPE(None, POINTER(pnanovdb_Compute), c_void_p, c_void_p, c_float, c_void_p, c_void_p, c_uint64, c_void_p),
        ),
        (
            "raster_to_nanovdb",
            CFUNCTYPE(
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_Compute),
                c_void_p,
                c_float,
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(pnanovdb_ComputeArray),
                POINTER(POINTER(pnanovdb_ComputeArray)),
                c_void_p,
                c_void_p,
            ),
        ),
        (
            "raster_file",
            CFUNCTYPE(
                c_int32,
                c_void_p,
                POINTER(pnanovdb_Compute),
                c_void_p,
                c_char_p,
                c_float,
                POINTER(POINTER(pnanovdb_ComputeArray)),
                POINTER(c_void_p),
                POINTER(c_void_p),
                POINTER(POINTER(pnanovdb_ComputeArray)),
                c_void_p,
                c_void_p,
                c_void_p,
            ),
        ),
        (
            "raster_to_nanovdb_from_arrays",
            CFUNCTYPE(
                c_int32,
                c_void_p,
                POINTER(pnanovdb_Compute),
                c_void_p,
                c_float,
                POINTER(POINTER(pnanovdb_ComputeArray)),
                c_uint32,
                POINTER(POINTER(pnanovdb_ComputeArray)),
            ),
        ),
        (
            "create_gaussian_data_from_arrays",
            CFUNCTYPE(
                c_int32,
                c_void_p,
                POINTER(pnanovdb_Compute),
                c_void_p,
                POINTER(POINTER(pnanovdb_ComputeArray)),
                c_uint32,
                POINTER(c_void_p),
                c_void_p,
                POINTER(c_void_p),
            ),
        ),
        ("create_gaussian_data_from_desc", c_void_p),
    ]


class Raster:
    """Python wrapper for pnanovdb_raster_t."""

    def __init__(self, compute: Compute, device=None):
        lib = load_library(COMPUTE_LIB)
        get_raster_func = lib.pnanovdb_get_raster
        get_raster_func.restype = POINTER(pnanovdb_Raster)
        get_raster_func.argtypes = []
        self._raster = get_raster_func()
        if not self._raster:
            raise RuntimeError("Failed to get raster")
        self._compute = compute
        self._compute_queue = compute.queue()
        self._raster.contents.compute = compute.get_compute()

    def raster_to_nanovdb(
        self,
        voxel_size: float,
        means: pnanovdb_ComputeArray,
        quaternions: pnanovdb_ComputeArray,
        scales: pnanovdb_ComputeArray,
        colors: pnanovdb_ComputeArray,
        sh_0: pnanovdb_ComputeArray,
        sh_n: pnanovdb_ComputeArray,
        opacities: pnanovdb_ComputeArray,
        shader_params_arrays=None,
        profiler_report=None,
        userdata=None,
    ) -> pnanovdb_ComputeArray:
        func = self._raster.contents.raster_to_nanovdb
        nanovdb_array = func(
            self._compute.get_compute(),
            self._compute_queue,
            voxel_size,
            pointer(means),
            pointer(quaternions),
            pointer(scales),
            pointer(colors),
            pointer(sh_0),
            pointer(sh_n),
            pointer(opacities),
            shader_params_arrays,
            profiler_report or c_void_p(),
            userdata or c_void_p(),
        )
        if not nanovdb_array:
            raise RuntimeError("Failed to raster points")
        return nanovdb_array.contents

    def raster_to_nanovdb_from_arrays(self, voxel_size: float, arrays) -> pnanovdb_ComputeArray:
        """Rasterize raw Gaussian arrays ``[means, opacities, quaternions, scales, sh_0, sh_n]``.

        The preprocessing of the reference (quaternion normalisation, scale
        exponentiation, SH0 -> colour, opacity sigmoid) runs inside the CUDA
        prep kernel; the caller's arrays are not modified.
        """
        if len(arrays) != 6:
            raise InvalidArgumentError(
                "Gaussian rasterization requires 6 arrays: [means, opacities, quaternions, scales, sh_0, sh_n]"
            )
        func = self._raster.contents.raster_to_nanovdb_from_arrays
        ArrayPtr = POINTER(pnanovdb_ComputeArray)
        arrays_c = (ArrayPtr * 6)(*[pointer(a) for a in arrays])
        out_array = ArrayPtr()
        ok = func(
            self._raster,
            self._compute.get_compute(),
            self._compute_queue,
            c_float(voxel_size),
            arrays_c,
            c_uint32(6),
            byref(out_array),
        )
        if not ok or not out_array:
            raise RuntimeError("Failed to rasterize Gaussian arrays to NanoVDB")
        return out_array.contents

    def raster_file(self, filename: str, voxel_size: float) -> pnanovdb_ComputeArray:
        func = self._raster.contents.raster_file
        out_array = POINTER(pnanovdb_ComputeArray)()
        ok = func(
            self._raster,
            self._compute.get_compute(),
            self._compute_queue,
            filename.encode("utf-8"),
            c_float(voxel_size),
            byref(out_array),
            None,
            None,
            None,
            None,
            None,
            None,
        )
        if not ok or not out_array:
            raise RuntimeError(f"Failed to rasterize {filename}")
        return out_array.contents

    def __del__(self):
        self._raster = None
        self._compute = None
