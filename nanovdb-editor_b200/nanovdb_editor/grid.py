"""Reader for the grid buffer the library returns.

Layout (``vox_grid_header_t`` in include/pnanovdb_b200.h): a 256-byte header,
the node2 region (root, then every node at its node2 size in node_idx order,
nanovdb_editor/PNanoVDBExt.h:28-83), the active-voxel bbox and per-value
arrays (RGBA8, float density, Vec3f colour) indexed by value index with two
background slots first.
"""

from __future__ import annotations

import numpy as np

HEADER_DTYPE = np.dtype(
    [
        ("magic", "<u8"),
        ("version", "<u4"),
        ("header_bytes", "<u4"),
        ("grid_bytes", "<u8"),
        ("node2_offset", "<u8"),
        ("node2_bytes", "<u8"),
        ("upper_count", "<u4"),
        ("lower_count", "<u4"),
        ("leaf_count", "<u4"),
        ("node_order", "<u4"),
        ("value_count", "<u8"),
        ("bbox_offset", "<u8"),
        ("rgba8_offset", "<u8"),
        ("density_offset", "<u8"),
        ("color_offset", "<u8"),
        ("voxel_size", "<f4"),
        ("bbox", "<i4", (6,)),
        ("pad0", "<u4"),
        ("pair_count", "<u8"),
        ("candidate_count", "<u8"),
        ("reserved", "u1", (112,)),
    ]
)
assert HEADER_DTYPE.itemsize == 256

GRID_MAGIC = 0x32454E58564F5642

# node2 word offsets (PNanoVDBExt.h:49-64)
OFF_VALUE_PREFIX = (258, 258, 34, 6)
OFF_VALUE_MASK = (386, 386, 50, 8)
OFF_CHILD_PREFIX = (898, 898, 114, 6)
OFF_CHILD_MASK = (1026, 1026, 130, 8)
OFF_CHILDREN = (2180, 1538, 194, 16)
NODE_BYTES = (541728, 274464, 34336, 128)


class NodeGrid:
    """Zero-copy numpy views over a grid buffer (bytes, bytearray or uint8 array)."""

    def __init__(self, buf):
        self.buf = np.frombuffer(buf, dtype=np.uint8) if not isinstance(buf, np.ndarray) else buf.view(np.uint8)
        self.header = self.buf[:256].view(HEADER_DTYPE)[0]
        if int(self.header["magic"]) != GRID_MAGIC:
            raise ValueError("not a voxel grid buffer (bad magic)")

    def _slice(self, off, count, dtype):
        dtype = np.dtype(dtype)
        return self.buf[int(off) : int(off) + int(count) * dtype.itemsize].view(dtype)

    @property
    def node2(self) -> np.ndarray:
        h = self.header
        return self.buf[int(h["node2_offset"]) : int(h["node2_offset"]) + int(h["node2_bytes"])]

    @property
    def value_count(self) -> int:
        return int(self.header["value_count"])

    @property
    def rgba8(self) -> np.ndarray:
        return self._slice(self.header["rgba8_offset"], self.value_count, np.uint32)

    @property
    def density(self) -> np.ndarray | None:
        """Float density per value index; None for a grid copied without the float channels."""
        off = self.header["density_offset"]
        return self._slice(off, self.value_count, np.float32) if off else None

    @property
    def color(self) -> np.ndarray | None:
        """Vec3f colour per value index; None for a grid copied without the float channels."""
        off = self.header["color_offset"]
        return self._slice(off, 3 * self.value_count, np.float32).reshape(-1, 3) if off else None

    @property
    def bbox(self) -> np.ndarray:
        return self._slice(self.header["bbox_offset"], 6, np.int32)

    @property
    def counts(self) -> dict:
        h = self.header
        return {
            "upper": int(h["upper_count"]),
            "lower": int(h["lower_count"]),
            "leaf": int(h["leaf_count"]),
            "voxels": self.value_count - 2,
            "pairs": int(h["pair_count"]),
            "candidates": int(h["candidate_count"]),
        }
