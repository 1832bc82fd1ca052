"""Builds libpnanovdbcompute.so (sm_100a) in-tree.

The library is the drop-in replacement of the reference's
``nanovdb_editor/lib/libpnanovdbcompute.so`` for the raster3d path; it is
written next to the Python package so ``nanovdb_editor.utils.load_library``
finds it the same way the reference's loader does.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB_DIR = os.path.join(HERE, "nanovdb_editor", "lib")
LIB = os.path.join(LIB_DIR, "libpnanovdbcompute.so")

SOURCES = ["vox_scan_sort.cu", "vox_raster.cu", "vox_leaf.cu", "vox_order.cu", "vox_backward.cu", "vox_api.cu", "vox_dropin.cu", "vox_noalloc.cu", "vox_voxelbvh.cu", "vox_optim.cu"]
NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)
    ]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", f"-I{INCLUDE}", f"-I{CSRC}", *sources(), "-lz", "-o", LIB]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
