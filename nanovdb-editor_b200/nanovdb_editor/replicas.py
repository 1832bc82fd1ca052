"""Host logic of multi-GPU runs: one process per GPU, each voxelizing its own
clouds (the path shards by independent clouds; no data-path collective).

* ``shard_clouds`` splits a batch of clouds into contiguous, Gaussian-balanced
  runs, one per rank (the batched form of `raster_gaussian_3d` over many clouds,
  raster/Raster.cpp:420-558, has no cross-cloud dependency).
* ``max_over_ranks`` is the job's time of a step: every rank waits for the
  slowest, so whole-job throughput divides the units all ranks processed by the
  maximum of the per-rank device times.
* ``job_rate`` is that throughput.

The process group is torch.distributed's (NCCL on GPUs, gloo on CPU); every
rank takes the same collective steps in the same order.
"""

from __future__ import annotations

import numpy as np


def shard_clouds(cloud_start, rank: int, world: int) -> tuple[int, int]:
    """Clouds [c0, c1) of `rank`: contiguous runs whose Gaussian counts are as
    even as whole clouds allow (boundaries at the cloud starts nearest to
    k * total / world).  Every cloud belongs to exactly one rank; a rank may get
    none when there are fewer clouds than ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    start = np.asarray(cloud_start, dtype=np.int64)
    if start.ndim != 1 or start.size < 1 or np.any(np.diff(start) < 0):
        raise ValueError("cloud_start must be a non-decreasing prefix of cloud sizes")
    n = start.size - 1
    total = int(start[-1] - start[0])
    targets = start[0] + (np.arange(world + 1, dtype=np.float64) * total / world)
    cuts = np.searchsorted(start, targets, side="left")
    cuts = np.clip(cuts, 0, n)
    cuts[0], cuts[-1] = 0, n
    cuts = np.maximum.accumulate(cuts)
    return int(cuts[rank]), int(cuts[rank + 1])


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar over the process group (the value itself
    without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """Sum of a per-rank scalar over the process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_all_ranks: float, max_ms: float) -> float:
    """Whole-job units per second: all ranks' units over the slowest rank's time."""
    if max_ms <= 0:
        raise ValueError("step time must be positive")
    return float(units_all_ranks) / (max_ms * 1e-3)
