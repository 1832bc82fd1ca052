"""B200 drop-in for nanovdb-editor's Gaussian -> NanoVDB voxelization path.

Mirrors the reference pymodule's raster3d surface (``nanovdb_editor.raster.Raster``,
``nanovdb_editor.compute.Compute``) over a CUDA implementation in
``lib/libpnanovdbcompute.so``, plus a differentiable ``voxelize`` op.
"""

from .compute import Compute, pnanovdb_ComputeArray  # noqa: F401
from .exceptions import InvalidArgumentError, PipelineError  # noqa: F401
from .grid import NodeGrid  # noqa: F401
from .raster import Raster, pnanovdb_Raster  # noqa: F401
