"""ctypes mirror of ``pnanovdb_compute_t`` (pymodule/nanovdb_editor/compute.py:42-217).

Only the parts the raster3d path uses are functional: arrays
(create / destroy / map / duplicate), load/save of grid buffers, and the
device/queue handles.  The structure layout matches the reference so the
reference's own binding code can read the table this library exports.
"""

from __future__ import annotations

from contextlib import contextmanager
from ctypes import (
    CFUNCTYPE,
    POINTER,
    Structure,
    c_byte,
    c_char_p,
    c_int,
    c_int32,
    c_size_t,
    c_uint32,
    c_uint64,
    c_void_p,
    cast,
    pointer,
)

import numpy as np

from .exceptions import InvalidArgumentError, PipelineError
from .utils import load_library

COMPUTE_LIB = "pnanovdbcompute"
pnanovdb_bool_t = c_int32


class pnanovdb_ComputeArray(Structure):
    """Definition equivalent to pnanovdb_compute_array_t (Compute.h:765-771)."""

    _fields_ = [("data", c_void_p), ("element_size", c_uint64), ("element_count", c_uint64), ("filepath", c_char_p)]


class pnanovdb_ShaderInterface(Structure):
    _fields_ = [("interface_pnanovdb_reflect_data_type", c_void_p), ("reserved", c_void_p * 3)]


class pnanovdb_DeviceInterface(Structure):
    """Compute.h:566-661 (34 pointers); unimplemented entries are NULL."""

    _fields_ = [
        ("interface_pnanovdb_reflect_data_type", c_void_p),
        ("create_device_manager", CFUNCTYPE(c_void_p, pnanovdb_bool_t)),
        ("destroy_device_manager", CFUNCTYPE(None, c_void_p)),
        ("enumerate_devices", CFUNCTYPE(pnanovdb_bool_t, c_void_p, c_uint32, c_void_p)),
        ("create_device", CFUNCTYPE(c_void_p, c_void_p, c_void_p)),
        ("destroy_device", CFUNCTYPE(None, c_void_p, c_void_p)),
        ("reserved_get_memory_stats", c_void_p),
        ("reserved_semaphore", c_void_p * 4),
        ("get_device_queue", CFUNCTYPE(c_void_p, c_void_p)),
        ("get_compute_queue", CFUNCTYPE(c_void_p, c_void_p)),
        ("flush", CFUNCTYPE(c_int, c_void_p, POINTER(c_uint64), c_void_p, c_void_p)),
        ("reserved_frames", c_void_p * 2),
        ("wait_idle", CFUNCTYPE(None, c_void_p)),
        ("reserved_interface", c_void_p * 2),
        ("reserved_swapchain", c_void_p * 5),
        ("reserved_encoder", c_void_p * 6),
        ("reserved_profiler", c_void_p * 3),
        ("get_device_index", CFUNCTYPE(c_uint32, c_void_p)),
    ]


class pnanovdb_Compute(Structure):
    """Definition equivalent to pnanovdb_compute_t (Compute.h:784-853)."""

    _fields_ = [
        ("interface_pnanovdb_reflect_data_type", c_void_p),
        ("module", c_void_p),
        ("compiler", c_void_p),
        ("shader_interface", pnanovdb_ShaderInterface),
        ("device_interface", pnanovdb_DeviceInterface),
        ("load_nanovdb", CFUNCTYPE(POINTER(pnanovdb_ComputeArray), c_char_p)),
        ("save_nanovdb", CFUNCTYPE(pnanovdb_bool_t, POINTER(pnanovdb_ComputeArray), c_char_p)),
        ("reserved_shader", c_void_p * 5),
        ("reserved_dispatch", c_void_p * 2),
        ("create_array", CFUNCTYPE(POINTER(pnanovdb_ComputeArray), c_size_t, c_uint64, c_void_p)),
        ("destroy_array", CFUNCTYPE(None, POINTER(pnanovdb_ComputeArray))),
        ("map_array", CFUNCTYPE(c_void_p, POINTER(pnanovdb_ComputeArray))),
        ("unmap_array", CFUNCTYPE(None, POINTER(pnanovdb_ComputeArray))),
        ("reserved_print_range", c_void_p),
        ("reserved_from_image", c_void_p),
        ("duplicate_array", CFUNCTYPE(POINTER(pnanovdb_ComputeArray), POINTER(pnanovdb_ComputeArray))),
    ]


class Compute:
    """Python wrapper for pnanovdb_compute_t (headless CUDA device)."""

    def __init__(self, compiler=None, device_index: int = 0):
        self._lib = load_library(COMPUTE_LIB)
        get_compute = self._lib.pnanovdb_get_compute
        get_compute.restype = POINTER(pnanovdb_Compute)
        get_compute.argtypes = []
        self._compute = get_compute()
        if not self._compute:
            raise PipelineError("Failed to get compute interface")
        self._compute.contents.module = self._lib._handle
        di = self._compute.contents.device_interface
        self._manager = di.create_device_manager(0)
        # pnanovdb_compute_device_desc_t (putil/Compute.h:503-508): device_index first
        desc = (c_uint32 * 4)(int(device_index), 0, 0, 0)
        # NULL without a CUDA device: the host-side array functions still work
        self._device = di.create_device(self._manager, cast(desc, c_void_p).value)
        self._queue = di.get_compute_queue(self._device)

    def get_compute(self):
        return self._compute

    def device(self):
        return self._device

    def queue(self):
        return self._queue

    def create_array(self, data: np.ndarray) -> pnanovdb_ComputeArray:
        data = np.ascontiguousarray(data)
        arr = self._compute.contents.create_array(data.itemsize, data.size, data.ctypes.data_as(c_void_p))
        if not arr:
            raise PipelineError("Failed to create compute array")
        return arr.contents

    def destroy_array(self, array: pnanovdb_ComputeArray) -> None:
        self._compute.contents.destroy_array(pointer(array))

    def duplicate_array(self, array: pnanovdb_ComputeArray) -> pnanovdb_ComputeArray:
        dup = self._compute.contents.duplicate_array(pointer(array))
        if not dup:
            raise PipelineError("Failed to duplicate compute array")
        return dup.contents

    def map_array(self, array: pnanovdb_ComputeArray, np_dtype) -> np.ndarray:
        np_dtype = np.dtype(np_dtype)
        if array.element_size * array.element_count % np_dtype.itemsize:
            raise InvalidArgumentError("Array size is not a multiple of the dtype size")
        ptr = self._compute.contents.map_array(pointer(array))
        if not ptr:
            raise PipelineError("Failed to map array")
        buf = (c_byte * (array.element_size * array.element_count)).from_address(ptr)
        return np.frombuffer(buf, dtype=np_dtype)

    def unmap_array(self, array: pnanovdb_ComputeArray) -> None:
        self._compute.contents.unmap_array(pointer(array))

    @contextmanager
    def mapped_array(self, array: pnanovdb_ComputeArray, np_dtype):
        view = self.map_array(array, np_dtype)
        try:
            yield view
        finally:
            self.unmap_array(array)

    def save_nanovdb(self, array: pnanovdb_ComputeArray, filepath: str) -> None:
        if not self._compute.contents.save_nanovdb(pointer(array), filepath.encode("utf-8")):
            raise PipelineError(f"Failed to save {filepath}")

    def load_nanovdb(self, filepath: str) -> pnanovdb_ComputeArray:
        arr = self._compute.contents.load_nanovdb(filepath.encode("utf-8"))
        if not arr:
            raise PipelineError(f"Failed to load NanoVDB file: {filepath}")
        return arr.contents

    def wait_idle(self) -> None:
        self._compute.contents.device_interface.wait_idle(self._queue)
