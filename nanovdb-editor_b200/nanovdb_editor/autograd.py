"""Differentiable voxelization as a torch.autograd.Function.

Forward: the library's voxelization with VOX_FLAG_DIFFERENTIABLE (the
reference's pair set and topology, raster/Raster.cpp:420-558, with the smooth
density / premultiplied colour channels).  Backward: ``vox_backward``, the
hand-written adjoint over the pair list.  Gradients are with respect to the
inputs as given: for ``raw=True`` (the reference's array form,
raster/RasterUtils.cpp:31-136) the raw quaternion, log-scales, opacity logits
and SH0 colours.
"""

from __future__ import annotations

import numpy as np
import torch

from .exceptions import PipelineError
from .grid import HEADER_DTYPE
from .vox import FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS, VoxContext

_NAMES = ("means", "quats", "scales", "opacities", "colors")


def _prep(t: torch.Tensor) -> torch.Tensor:
    if not t.is_cuda:
        raise PipelineError("voxelize: inputs must be CUDA tensors")
    return t.detach().to(torch.float32).contiguous()


class VoxelizeFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, quats, scales, opacities, colors, voxel_size, raw, vox):
        ins = [_prep(t) for t in (means, quats, scales, opacities, colors)]
        torch.cuda.current_stream(ins[0].device).synchronize()  # the library reads on its own stream
        flags = FLAG_DIFFERENTIABLE | (FLAG_RAW_INPUTS if raw else 0)
        _, nbytes = vox.voxelize(*ins, float(voxel_size), 0.05, flags)
        grid = torch.empty(nbytes, dtype=torch.uint8, device=ins[0].device)
        vox.grid_device(grid)
        h = np.frombuffer(grid[:256].cpu().numpy().tobytes(), HEADER_DTYPE)[0]
        vc = int(h["value_count"])
        d0, c0 = int(h["density_offset"]), int(h["color_offset"])
        density = grid[d0 : d0 + 4 * vc].view(torch.float32).clone()
        color = grid[c0 : c0 + 12 * vc].view(torch.float32).view(vc, 3).clone()
        ctx.save_for_backward(*ins)
        ctx.vox = vox
        ctx.generation = vox.generation
        ctx.mark_non_differentiable(grid)
        return density, color, grid

    @staticmethod
    def backward(ctx, g_density, g_color, _g_grid):
        vox: VoxContext = ctx.vox
        if vox.generation != ctx.generation:
            raise PipelineError("voxelize backward: the context ran another voxelization after this forward; "
                                "use one context per differentiable graph")
        ins = ctx.saved_tensors
        gd = None if g_density is None else g_density.detach().to(torch.float32).contiguous()
        gc = None if g_color is None else g_color.detach().to(torch.float32).contiguous()
        out = {k: torch.empty_like(t) for k, t, need in zip(_NAMES, ins, ctx.needs_input_grad[:5]) if need}
        torch.cuda.current_stream(ins[0].device).synchronize()
        vox.backward(*ins, gd, gc, out)
        return tuple(out.get(k) for k in _NAMES) + (None, None, None)


_CONTEXTS: dict[int, VoxContext] = {}


def default_context(device: int = 0) -> VoxContext:
    if device not in _CONTEXTS:
        _CONTEXTS[device] = VoxContext(device)
    return _CONTEXTS[device]


def voxelize(means, quats, scales, opacities, colors, voxel_size: float, raw: bool = True, context: VoxContext | None = None):
    """Differentiable voxelization of CUDA tensors.

    Returns (density [value_count], colour [value_count, 3], grid) where
    density / colour carry gradients (value index order, two background slots
    first) and grid is the library's grid buffer as a CUDA uint8 tensor.
    """
    vox = context or default_context(means.device.index or 0)
    return VoxelizeFunction.apply(means, quats, scales, opacities, colors, float(voxel_size), bool(raw), vox)


def voxel_coords(vox: VoxContext, value_count: int, device) -> torch.Tensor:
    """(i, j, k) of the active voxels of the context's last (single-cloud) grid, row r = value index r + 2."""
    out = torch.full((max(int(value_count), 2), 3), -(1 << 31), dtype=torch.int32, device=device)
    if value_count > 2:
        vox.voxel_coords(out)
    return out[2:]


def pack_coords(ijk: torch.Tensor) -> torch.Tensor:
    """int64 keys of (i, j, k) in [-2^20, 2^20) for matching voxels of two grids."""
    b = ijk.to(torch.int64) + (1 << 20)
    return (b[:, 0] << 42) | (b[:, 1] << 21) | b[:, 2]


class TargetGrid:
    """Density of a fixed grid, looked up by voxel coordinate (0 where inactive)."""

    def __init__(self, coords: torch.Tensor, density: torch.Tensor):
        keys = pack_coords(coords)
        order = torch.argsort(keys)
        self.keys = keys[order].contiguous()
        self.density = density[order].contiguous()
        self.total_sq = float((self.density.double() ** 2).sum())

    @classmethod
    def from_last(cls, vox: VoxContext, density: torch.Tensor) -> "TargetGrid":
        """From the context's last grid and its density channel (value index order)."""
        coords = voxel_coords(vox, density.shape[0], density.device)
        return cls(coords, density[2:].detach())

    def lookup(self, coords: torch.Tensor):
        k = pack_coords(coords)
        if self.keys.numel() == 0:
            return torch.zeros(k.shape, dtype=torch.float32, device=k.device), torch.zeros(k.shape, dtype=torch.bool, device=k.device)
        pos = torch.searchsorted(self.keys, k).clamp(max=self.keys.numel() - 1)
        hit = self.keys[pos] == k
        return torch.where(hit, self.density[pos], torch.zeros((), device=k.device)), hit


def l2_to_target(density: torch.Tensor, vox: VoxContext, target: TargetGrid) -> torch.Tensor:
    """0.5 * sum over the union of both grids' voxels of (density - target)^2.

    `density` must come from the context's last voxelization (its voxel
    coordinates are read from the context)."""
    coords = voxel_coords(vox, density.shape[0], density.device)
    t, _ = target.lookup(coords)
    d = density[2:]
    missing = target.total_sq - float((t.double() ** 2).sum())  # target voxels the grid lacks: constant
    return 0.5 * ((d - t) ** 2).sum() + 0.5 * missing
