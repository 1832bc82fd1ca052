"""Native library loading (mirrors pymodule/nanovdb_editor/utils.py:67-83).

The library lives in ``nanovdb_editor/lib`` next to this package.  There is
no fallback: if the CUDA library is missing the import of the raster API
fails loudly.
"""

from __future__ import annotations

import ctypes
import os

_LIBS = {}


def lib_dir() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")


def load_library(lib_name: str) -> ctypes.CDLL:
    path = os.path.join(lib_dir(), f"lib{lib_name}.so")
    if path not in _LIBS:
        if not os.path.exists(path):
            raise OSError(
                f"{path} not found: build it with nanovdb-editor_b200/build_ext.py (nvcc, sm_100a)"
            )
        _LIBS[path] = ctypes.CDLL(path)
    return _LIBS[path]
