"""The reference's own Python binding, unchanged, against this library (CPU).

The reference's pymodule (pymodule/nanovdb_editor/raster.py, compute.py,
device.py) is imported as it ships, from a temporary copy whose lib/ folder
holds this library in place of the reference's libpnanovdbcompute.so:

* its ctypes structures (pnanovdb_Raster, pnanovdb_Compute,
  pnanovdb_DeviceInterface, pnanovdb_ComputeArray) have, field for field, the
  offsets include/pnanovdb_b200.h gives the same fields (the reference's
  Python raster table stops before create_gaussian_data_from_desc: a prefix);
* its DeviceInterface class finds this library's device interface and creates
  a device manager;
* its pnanovdb_Compute / pnanovdb_Raster structures, bound to this library's
  tables, create, map, duplicate and destroy arrays and run the table entries
  that need no GPU (create_gaussian_data_from_arrays without a context,
  destroy_gaussian_data, the argument checks of
  raster_to_nanovdb_from_arrays), with the reference's own CFUNCTYPE
  signatures.

The voxelizing entries need a GPU; the GPU tests call them through
nanovdb_editor/raster.py, whose structures this test shows to be
layout-identical to the reference's.  Skipped when the reference checkout is
absent.
"""

import json
import os
import shutil
import subprocess
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "nanovdb-editor_b200", "nanovdb_editor", "lib", "libpnanovdbcompute.so")
REFERENCE = os.environ.get("VOX_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
PYMODULE = os.path.join(REFERENCE, "pymodule", "nanovdb_editor")

CHILD = r"""
import ctypes, json, sys
import numpy as np
import nanovdb_editor.raster as R
import nanovdb_editor.compute as C
import nanovdb_editor.device as D

def offsets(cls):
    return {name: getattr(cls, name).offset for name, _ in cls._fields_}

out = {
    "raster": offsets(R.pnanovdb_Raster), "raster_size": ctypes.sizeof(R.pnanovdb_Raster),
    "compute": offsets(C.pnanovdb_Compute), "compute_size": ctypes.sizeof(C.pnanovdb_Compute),
    "device": offsets(D.pnanovdb_DeviceInterface), "device_size": ctypes.sizeof(D.pnanovdb_DeviceInterface),
    "array": offsets(C.pnanovdb_ComputeArray), "array_size": ctypes.sizeof(C.pnanovdb_ComputeArray),
}

lib = ctypes.CDLL(sys.argv[1])
get_raster = lib.pnanovdb_get_raster
get_raster.restype = ctypes.POINTER(R.pnanovdb_Raster)
rp = get_raster()
r = rp.contents
out["raster_entries"] = [name for name, _ in R.pnanovdb_Raster._fields_[2:]
                         if ctypes.cast(getattr(r, name), ctypes.c_void_p).value]

di = D.DeviceInterface(0)  # the reference's class, this library's device interface
di.create_device_manager()
out["device_manager"] = True

get_compute = lib.pnanovdb_get_compute
get_compute.restype = ctypes.POINTER(C.pnanovdb_Compute)
cp = get_compute()
comp = cp.contents
x = np.arange(12, dtype=np.float32)
arr = comp.create_array(4, 12, x.ctypes.data)
ptr = comp.map_array(arr)
got = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), shape=(12,)).copy()
comp.unmap_array(arr)
dup = comp.duplicate_array(arr)
out["array_roundtrip"] = bool(np.array_equal(got, x)) and dup.contents.element_count == 12
comp.destroy_array(dup)
comp.destroy_array(arr)

# Gaussian data from raw arrays [means, opacities, quats, scales, sh_0] (no context: host only)
n = 5
rng = np.random.default_rng(0)
raw = [rng.normal(size=(n, 3)), rng.normal(size=n), rng.normal(size=(n, 4)), rng.normal(size=(n, 3)) - 4,
       rng.normal(size=(n, 3))]
raw = [np.ascontiguousarray(a, np.float32) for a in raw]
cas = [comp.create_array(4, a.size, a.ctypes.data) for a in raw]
Arr = ctypes.POINTER(C.pnanovdb_ComputeArray)
arrays = (Arr * 5)(*cas)
gdata = ctypes.c_void_p()
ok = r.create_gaussian_data_from_arrays(rp, cp, None, arrays, 5, ctypes.byref(gdata), None, None)
out["create_from_arrays"] = [int(ok), bool(gdata.value)]
r.destroy_gaussian_data(cp, None, gdata)
result = Arr()
ok = r.raster_to_nanovdb_from_arrays(rp, cp, None, ctypes.c_float(0.1), arrays, 4, ctypes.byref(result))
out["from_arrays_too_few"] = [int(ok), bool(result)]
for a in cas:
    comp.destroy_array(a)
print(json.dumps(out))
"""

C_OFFSETS = r"""
#include <stdio.h>
#include <stddef.h>
#include "pnanovdb_b200.h"
#define P(t, f) printf("%s %s %zu\n", #t, #f, offsetof(t, f));
int main(void) {
@FIELDS@
  printf("size raster %zu\nsize compute %zu\nsize device %zu\nsize array %zu\n", sizeof(pnanovdb_raster_t),
         sizeof(pnanovdb_compute_t), sizeof(pnanovdb_compute_device_interface_t), sizeof(pnanovdb_compute_array_t));
  return 0;
}
"""

STRUCTS = {
    "raster": "pnanovdb_raster_t",
    "compute": "pnanovdb_compute_t",
    "device": "pnanovdb_compute_device_interface_t",
    "array": "pnanovdb_compute_array_t",
}


@pytest.fixture(scope="module")
def ref_binding():
    if not os.path.isdir(PYMODULE):
        pytest.skip("reference checkout not found (set VOX_REFERENCE_DIR)")
    if not os.path.exists(LIB):
        import build_ext

        build_ext.build()
    with tempfile.TemporaryDirectory() as d:
        pkg = os.path.join(d, "nanovdb_editor")
        shutil.copytree(PYMODULE, pkg)
        os.makedirs(os.path.join(pkg, "lib"), exist_ok=True)
        os.symlink(LIB, os.path.join(pkg, "lib", "libpnanovdbcompute.so"))
        env = dict(os.environ, PYTHONPATH=d)
        p = subprocess.run([sys.executable, "-c", CHILD, LIB], cwd=d, env=env, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-3000:]
        yield json.loads(p.stdout.strip().splitlines()[-1])


def header_offsets(names):
    """offsetof() of the given fields in include/pnanovdb_b200.h, and the struct sizes."""
    lines = "".join(f"  P({STRUCTS[k]}, {f})\n" for k, fs in names.items() for f in fs)
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "o.c"), os.path.join(d, "o")
        open(src, "w").write(C_OFFSETS.replace("@FIELDS@", lines))
        subprocess.run(["gcc", "-I", INCLUDE, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    offs, sizes = {}, {}
    for line in out:
        parts = line.split()
        if len(parts) == 3 and parts[0] == "size":
            sizes[parts[1]] = int(parts[2])
        elif len(parts) == 3:
            offs[(parts[0], parts[1])] = int(parts[2])
    return offs, sizes


# fields this library's header names (the others are reserved slots of the same size)
NAMED = {
    "raster": None,  # every field of the reference's Python raster table
    "compute": ["interface_pnanovdb_reflect_data_type", "module", "compiler", "shader_interface", "device_interface",
                "load_nanovdb", "save_nanovdb", "create_array", "destroy_array", "map_array", "unmap_array",
                "duplicate_array"],
    "device": ["interface_pnanovdb_reflect_data_type", "create_device_manager", "destroy_device_manager",
               "enumerate_devices", "create_device", "destroy_device", "get_device_queue", "get_compute_queue",
               "flush", "wait_idle", "get_device_index"],
    "array": ["data", "element_size", "element_count", "filepath"],
}


def test_reference_ctypes_layouts_match_header(ref_binding):
    names = {k: (list(ref_binding[k]) if v is None else v) for k, v in NAMED.items()}
    offs, sizes = header_offsets(names)
    for k, fields in names.items():
        for f in fields:
            assert offs[(STRUCTS[k], f)] == ref_binding[k][f], (k, f)
    assert sizes["compute"] == ref_binding["compute_size"]
    assert sizes["device"] == ref_binding["device_size"]
    assert sizes["array"] == ref_binding["array_size"] == 32
    # the reference's Python raster table is a prefix of the C table (it omits create_gaussian_data_from_desc)
    assert ref_binding["raster_size"] == sizes["raster"] - 8


def test_reference_binding_drives_the_tables(ref_binding):
    assert ref_binding["device_manager"] is True
    assert set(ref_binding["raster_entries"]) == set(list(ref_binding["raster"])[2:])  # every entry bound, non-NULL
    assert ref_binding["array_roundtrip"] is True
    assert ref_binding["create_from_arrays"] == [1, True]
    assert ref_binding["from_arrays_too_few"] == [0, False]  # fewer than 5 arrays: FALSE, no result
