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
from .vox import FLAG_BF16_INPUTS, FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS, VoxContext

_NAMES = ("means", "quats", "scales", "opacities", "colors")


def _prep(t: torch.Tensor, bf16: bool) -> torch.Tensor:
    if not t.is_cuda:
        raise PipelineError("voxelize: inputs must be CUDA tensors")
    return t.detach().to(torch.bfloat16 if bf16 else torch.float32).contiguous()


class VoxelizeFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, quats, scales, opacities, colors, voxel_size, raw, vox):
        # bfloat16 attributes (all five) are read as such (VOX_FLAG_BF16_INPUTS); gradients are FP32
        bf16 = all(t.dtype == torch.bfloat16 for t in (means, quats, scales, opacities, colors))
        ins = [_prep(t, bf16) for t in (means, quats, scales, opacities, colors)]
        torch.cuda.current_stream(ins[0].device).synchronize()  # the library reads on its own stream
        flags = FLAG_DIFFERENTIABLE | (FLAG_RAW_INPUTS if raw else 0) | (FLAG_BF16_INPUTS if bf16 else 0)
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
        out = {k: torch.empty(t.shape, dtype=torch.float32, device=t.device)
               for k, t, need in zip(_NAMES, ins, ctx.needs_input_grad[:5]) if need}
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


def batch_voxel_keys(vox: VoxContext, value_offsets, device):
    """int64 keys (cloud, i, j, k) of every value index of the context's last
    batched grid (clouds back to back), and a mask that is False on each
    cloud's two background slots."""
    voff = torch.as_tensor(np.asarray(value_offsets, dtype=np.int64), device=device)
    total = int(voff[-1])
    ijk = torch.full((max(total, 1), 3), -(1 << 31), dtype=torch.int32, device=device)
    if total:
        vox.voxel_coords(ijk)
    ijk = ijk[:total]
    counts = voff[1:] - voff[:-1]
    cloud = torch.repeat_interleave(torch.arange(counts.numel(), device=device), counts)
    local = torch.arange(total, device=device) - voff[:-1][cloud]
    valid = local >= 2
    b = ijk.to(torch.int64) + (1 << 18)  # |coordinate| < 2^17 (the node2 root key range)
    keys = (cloud << 57) | (b[:, 0] << 38) | (b[:, 1] << 19) | b[:, 2]
    return keys, valid


class BatchTargetGrid:
    """Per-cloud target densities of a batched grid, looked up by (cloud, voxel)."""

    def __init__(self, keys: torch.Tensor, valid: torch.Tensor, density: torch.Tensor):
        k = keys[valid]
        d = density[valid].detach()
        order = torch.argsort(k)
        self.keys = k[order].contiguous()
        self.density = d[order].contiguous()
        self.total_sq = float((self.density.double() ** 2).sum())

    def lookup(self, keys: torch.Tensor):
        if self.keys.numel() == 0:
            return torch.zeros(keys.shape, dtype=torch.float32, device=keys.device)
        pos = torch.searchsorted(self.keys, keys).clamp(max=self.keys.numel() - 1)
        return torch.where(self.keys[pos] == keys, self.density[pos], torch.zeros((), device=keys.device))


def l2_to_batch_target(density: torch.Tensor, keys: torch.Tensor, valid: torch.Tensor, target: BatchTargetGrid):
    """0.5 * sum over every cloud's voxels (the union with its target's) of
    (density - target)^2, and dL/d density (zero on background slots)."""
    t = target.lookup(keys)
    diff = torch.where(valid, density - t, torch.zeros((), device=density.device))
    missing = target.total_sq - float((torch.where(valid, t, torch.zeros((), device=t.device)).double() ** 2).sum())
    return 0.5 * float((diff.double() ** 2).sum()) + 0.5 * missing, diff
