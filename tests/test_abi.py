"""C-ABI checks that need no GPU: the library loads, exports every function
include/*.h declares, and its table layouts match both the header and the
reference's ctypes binding (pymodule/nanovdb_editor/raster.py:14-168,
compute.py:109-217)."""

import ctypes
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "nanovdb-editor_b200", "nanovdb_editor", "lib", "libpnanovdbcompute.so")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import build_ext

        build_ext.build()
    return ctypes.CDLL(LIB)


def declared_functions():
    names = []
    for f in sorted(os.listdir(INCLUDE)):
        if not f.endswith(".h") or f == "vox_detmath.h":
            continue
        src = open(os.path.join(INCLUDE, f)).read()
        names += re.findall(r"^PNANOVDB_API\s+[^;(]*?\b(\w+)\s*\(", src, flags=re.M)
    return names


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert "pnanovdb_get_raster" in names and "vox_voxelize" in names
    for n in names:
        assert hasattr(lib, n), n


def test_tables_without_gpu(lib):
    from nanovdb_editor.compute import Compute, pnanovdb_Compute
    from nanovdb_editor.raster import pnanovdb_Raster

    get_raster = lib.pnanovdb_get_raster
    get_raster.restype = ctypes.POINTER(pnanovdb_Raster)
    r = get_raster()
    assert r and r.contents.raster_to_nanovdb and r.contents.raster_to_nanovdb_from_arrays
    assert r.contents.raster_gaussian_3d and r.contents.raster_file
    c = Compute()
    arr = c.create_array(__import__("numpy").arange(10, dtype="float32"))
    assert arr.element_count == 10 and arr.element_size == 4
    view = c.map_array(arr, "float32")
    assert float(view[3]) == 3.0
    c.destroy_array(arr)
    assert ctypes.sizeof(pnanovdb_Compute) > 0


C_LAYOUT = r"""
#include <stdio.h>
#include <stddef.h>
#include "pnanovdb_b200.h"
int main(void) {
  printf("raster %zu %zu %zu %zu\n", sizeof(pnanovdb_raster_t), offsetof(pnanovdb_raster_t, raster_gaussian_3d),
         offsetof(pnanovdb_raster_t, raster_to_nanovdb_from_arrays), offsetof(pnanovdb_raster_t, create_gaussian_data_from_desc));
  printf("compute %zu %zu %zu %zu\n", sizeof(pnanovdb_compute_t), offsetof(pnanovdb_compute_t, create_array),
         offsetof(pnanovdb_compute_t, duplicate_array), sizeof(pnanovdb_compute_device_interface_t));
  printf("array %zu\nheader %zu\n", sizeof(pnanovdb_compute_array_t), sizeof(vox_grid_header_t));
  return 0;
}
"""


def test_struct_layouts_match_header():
    from nanovdb_editor.compute import pnanovdb_Compute, pnanovdb_ComputeArray, pnanovdb_DeviceInterface
    from nanovdb_editor.grid import HEADER_DTYPE
    from nanovdb_editor.raster import pnanovdb_Raster

    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(src, "w").write(C_LAYOUT)
        subprocess.run(["gcc", "-I", INCLUDE, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    raster = [int(x) for x in out[0].split()[1:]]
    compute = [int(x) for x in out[1].split()[1:]]
    assert raster == [
        ctypes.sizeof(pnanovdb_Raster),
        pnanovdb_Raster.raster_gaussian_3d.offset,
        pnanovdb_Raster.raster_to_nanovdb_from_arrays.offset,
        pnanovdb_Raster.create_gaussian_data_from_desc.offset,
    ]
    # reference layout: reflect + compute + 12 function pointers
    assert raster[0] == 14 * 8 and raster[1] == 8 * 8
    assert compute == [
        ctypes.sizeof(pnanovdb_Compute),
        pnanovdb_Compute.create_array.offset,
        pnanovdb_Compute.duplicate_array.offset,
        ctypes.sizeof(pnanovdb_DeviceInterface),
    ]
    # Compute.h:784-853: reflect, module, compiler, shader iface (4 ptrs),
    # device iface (34 ptrs), then load/save + 7 shader/dispatch entries
    assert compute[3] == 34 * 8 and compute[1] == (3 + 4 + 34 + 2 + 7) * 8
    assert int(out[2].split()[1]) == ctypes.sizeof(pnanovdb_ComputeArray) == 32
    assert int(out[3].split()[1]) == HEADER_DTYPE.itemsize == 256
