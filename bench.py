"""Benchmark: Gaussian -> NanoVDB (node2) voxelization on B200.

Workload (one step = one full voxelization of one cloud): 2M Gaussians drawn
from 64 surface-like clusters (cluster_cloud), voxel size 0.002, float32
attributes in the raw on-disk convention (log scales, logit opacities, SH0).
Data: seeded synthetic (the reference publishes no dataset for this path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value   Gaussians/s with inputs resident in HBM (vox_voxelize on device
        pointers), per-step CUDA events on the library's stream, L2 flushed
        between steps; whole job over N ranks (weak scaling: each rank
        voxelizes its own cloud).
e2e     same metric through the reference-facing C ABI with host buffers
        (pnanovdb_raster_t.raster_to_nanovdb_from_arrays: pinned host inputs
        in, host grid out, copies inside the timed call).
roofline  achieved HBM GB/s of the dominant kernel (the leaf walk) from the
        algorithmic bytes of the (voxel, Gaussian)-pair work it performs - emit
        12 B/pair (8 B key + 4 B id), sort 24 B/pair per 8-bit pass over the
        voxel keys, accumulate 12 B/pair, values 20 B/voxel - and its
        CUDA-event duration, against MEASURED_PEAKS.json; beside it the same
        figure for the whole step (plus 2 x 56 B attribute reads per Gaussian
        and the topology bytes), the kernel's own byte count, and the DRAM
        traffic ncu measured for it.
cpu_baseline  the CPU oracle (C restatement of the reference path; the
        reference's Vulkan path is unavailable on this box) on a bounded
        sample of the same workload on all host cores.
--impl reference  times that CPU implementation alone (rank 0).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "nanovdb-editor_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Gaussians/s voxelized: plain vs batched vs fwd+bwd at 1e-5 rel; % of HBM peak"
UNIT = "Gaussians/s"
WORKLOAD = {"workload": "plain_forward_2M_clusters64_vs0.002", "gaussians": 2_000_000, "clusters": 64, "voxel_size": 0.002}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index=0):
        self.proc = None
        self.out = []
        self.device_index = device_index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL,
                text=True,
            )
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def run_config(G, world):
    """The workload config both arms report (the CPU arm times a stated sample of it)."""
    return dict(WORKLOAD, gaussians=G, parallelism=f"replicas{world}" if world > 1 else "single",
                l2="256 MB flush between steps; pair working set >> L2", inputs="raw (log-scale, logit, SH0)")


def cpu_baseline(steps=1, target_s=15.0):
    """Oracle (float outputs only) on a bounded sample of the workload, all host cores."""
    import oracle as oracle_py
    from nanovdb_editor import workloads as W

    oracle_py.build()
    cores = os.cpu_count() or 1
    vs = WORKLOAD["voxel_size"]
    n = 20_000
    rate = None
    sample = None
    counts = {}
    dt = 0.0
    for _ in range(4):
        # clusters of the 2M workload's size (31,250 Gaussians), so the sample has its density
        clusters = max(1, round(n / 31_250))
        cloud = W.cluster_cloud(n, 1, clusters=clusters)
        t0 = time.perf_counter()
        r = oracle_py.OracleResult(cloud, vs, 0.05, window_mode=1 | 2, nthreads=cores)
        dt = time.perf_counter() - t0
        ok = r.counts["error"] == 0
        counts = dict(r.counts)
        r.close()
        rate = n / dt if ok else None
        sample = (f"a sample of the workload: {n} Gaussians in {clusters} cluster(s) of the 2M workload's "
                  f"distribution and per-cluster density, voxel 0.002, {dt:.1f}s")
        if dt > target_s / 4 or n >= 400_000:
            break
        n = int(min(400_000, n * max(2.0, target_s / max(dt, 1e-3) / 2)))
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
            "pairs_per_s": counts.get("P", 0) / dt if dt else None, "voxels_per_s": counts.get("V", 0) / dt if dt else None}


CFG0 = {"workload": "cfg0_plain_100k_vs0.01", "gaussians": 100_000, "voxel_size": 0.01}


def cpu_cfg0():
    """The reference's CPU-runnable configuration (100K Gaussians, uniform in
    [-1, 1]^3, voxel 0.01) voxelized in full by the CPU restatement in the
    reference's fragment windows, on all host cores."""
    import oracle as oracle_py
    from nanovdb_editor import workloads as W

    oracle_py.build()
    cores = os.cpu_count() or 1
    cloud = W.plain_cloud(CFG0["gaussians"], 0)
    t0 = time.perf_counter()
    r = oracle_py.OracleResult(cloud, CFG0["voxel_size"], 0.05, window_mode=1 | 2, nthreads=cores)
    dt = time.perf_counter() - t0
    c = dict(r.counts)
    r.close()
    return dict(CFG0, cores=cores, seconds=dt, gaussians_per_s=CFG0["gaussians"] / dt, pairs_per_s=c["P"] / dt,
                voxels_per_s=c["V"] / dt, windows=c["windows"])


def gpu_cfg0(ctx, torch, steps, warmup, flush):
    """The same configuration on the GPU through raster_to_nanovdb-style device
    inputs (activated arrays, the reference's node order), CUDA events."""
    from nanovdb_editor import workloads as W
    from nanovdb_editor.vox import FLAG_WINDOW_ORDER

    cloud = W.plain_cloud(CFG0["gaussians"], 0)
    dev = [torch.from_numpy(np.ascontiguousarray(cloud[k])).cuda() for k in ("means", "quats", "scales", "opacities", "colors")]
    ext = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(warmup):
        ctx.voxelize(*dev, CFG0["voxel_size"], 0.05, FLAG_WINDOW_ORDER)
    ts = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0.record(ext)
        ctx.voxelize(*dev, CFG0["voxel_size"], 0.05, FLAG_WINDOW_ORDER)
        e1.record(ext)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    st = ctx.stats()
    ms = float(np.mean(ts))
    return dict(CFG0, ms_per_step=ms, gaussians_per_s=CFG0["gaussians"] / (ms * 1e-3), pairs_per_s=st["pairs"] / (ms * 1e-3),
                voxels_per_s=st["voxels"] / (ms * 1e-3), node_order="reference (window order)")


FWD_BWD = {"workload": "fwd_bwd_500k_clusters64_vs0.004", "gaussians": 500_000, "clusters": 64, "voxel_size": 0.004}


def measure_fwd_bwd(ctx, torch, rank, steps, warmup, flush):
    """Plain forward vs forward + adjoint on the 500K-Gaussian differentiable
    workload (cluster distribution, voxel 0.004), upstream dL/dvoxel ~ N(0, 1)
    on the active voxels; CUDA events on the library's stream, L2 flushed."""
    from nanovdb_editor import workloads as W
    from nanovdb_editor.vox import FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS

    G = FWD_BWD["gaussians"]
    vs = FWD_BWD["voxel_size"]
    raw = W.cluster_cloud(G, 101 + rank, clusters=FWD_BWD["clusters"]).raw_arrays()
    dev = [torch.from_numpy(a).cuda() for a in raw[:5]]
    ins = (dev[0], dev[2], dev[3], dev[1], dev[4])  # means, quats, log scales, logits, SH0
    out = {k: torch.empty_like(t) for k, t in zip(("means", "quats", "scales", "opacities", "colors"), ins)}
    ext = torch.cuda.ExternalStream(ctx.stream)
    ev0, ev1, ev2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    ctx.voxelize(*ins, vs, 0.05, FLAG_RAW_INPUTS | FLAG_DIFFERENTIABLE)
    vc = int(ctx.stats()["value_count"])
    gen = torch.Generator(device="cuda").manual_seed(7)
    gd = torch.randn(vc, device="cuda", generator=gen)
    gc = torch.randn((vc, 3), device="cuda", generator=gen)
    gd[:2] = 0
    gc[:2] = 0
    torch.cuda.synchronize()

    def timed(fn):
        for _ in range(warmup):
            fn()
        res = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0.record(ext)
            fn()
            ev2.record(ext)
            ev2.synchronize()
            res.append(ev0.elapsed_time(ev2))
        return float(np.mean(res))

    plain_ms = timed(lambda: ctx.voxelize(*ins, vs, 0.05, FLAG_RAW_INPUTS))
    fwd_ms = timed(lambda: ctx.voxelize(*ins, vs, 0.05, FLAG_RAW_INPUTS | FLAG_DIFFERENTIABLE))
    bwd_only = []

    def fwd_bwd():
        ctx.voxelize(*ins, vs, 0.05, FLAG_RAW_INPUTS | FLAG_DIFFERENTIABLE)
        ctx.backward(*ins, gd, gc, out)
        bwd_only.append(ctx.stats()["ms_backward"])

    fb_ms = timed(fwd_bwd)
    st = ctx.stats()
    return {
        "workload": FWD_BWD["workload"],
        "gaussians": G,
        "pairs": int(st["pairs"]),
        "voxels": int(st["voxels"]),
        "plain_forward_ms": plain_ms,
        "differentiable_forward_ms": fwd_ms,
        "backward_ms": float(np.mean(bwd_only[-steps:])),
        "fwd_bwd_ms": fb_ms,
        "fwd_bwd_over_plain": fb_ms / plain_ms,
        "fwd_bwd_gaussians_per_s": G / (fb_ms * 1e-3),
        "plain_gaussians_per_s": G / (plain_ms * 1e-3),
        "tolerance": "1e-5 of each gradient family's max vs the FP64 adjoint (tests/test_gpu_adjoint.py)",
    }


BATCHED = {"workload": "batched_256_clouds_1k-200k_vs0.002-0.02", "clouds": 256, "min_n": 1_000, "max_n": 200_000}


def measure_batched(ctx, torch, rank, steps, warmup, flush):
    """Uneven batch (256 clouds, log-uniform 1k-200k Gaussians, 1-16 clusters,
    voxel size log-uniform in [0.002, 0.02]): one vox_voxelize_batch call vs the
    plain form, one vox_voxelize call per cloud back to back; inputs resident in
    HBM, CUDA events on the library's stream around the whole batch."""
    from nanovdb_editor import workloads as W
    from nanovdb_editor.vox import FLAG_RAW_INPUTS

    clouds, start, vs = W.batch_clouds(BATCHED["clouds"], 3 + rank, BATCHED["min_n"], BATCHED["max_n"])
    allc = W.concat(clouds)
    raw = allc.raw_arrays()
    dev = [torch.from_numpy(a).cuda() for a in raw[:5]]
    ins = (dev[0], dev[2], dev[3], dev[1], dev[4])
    G = int(start[-1])
    ext = torch.cuda.ExternalStream(ctx.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(warmup):
            fn()
        res = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            ev0.record(ext)
            fn()
            ev1.record(ext)
            ev1.synchronize()
            res.append(ev0.elapsed_time(ev1))
        return float(np.mean(res))

    def batched():
        ctx.voxelize_batch(*ins, start, vs, 0.05, FLAG_RAW_INPUTS)

    views = [tuple(t[int(a):int(b)] for t in ins) for a, b in zip(start[:-1], start[1:])]

    def plain():
        for v, x in zip(views, vs):
            ctx.voxelize(*v, float(x), 0.05, FLAG_RAW_INPUTS)

    b_ms = timed(batched)
    st = ctx.stats()
    p_ms = timed(plain)
    return {
        "workload": BATCHED["workload"],
        "clouds": len(clouds),
        "gaussians": G,
        "pairs": int(st["pairs"]),
        "voxels": int(st["voxels"]),
        "batched_ms": b_ms,
        "plain_loop_ms": p_ms,
        "batched_gaussians_per_s": G / (b_ms * 1e-3),
        "plain_loop_gaussians_per_s": G / (p_ms * 1e-3),
        "batched_over_plain": p_ms / b_ms,
        "parity": "every cloud's grid byte-identical to its single-cloud grid (tests/test_gpu_batch.py)",
    }


def measure_batched_fwd_bwd(ctx, torch, rank, steps, warmup, flush):
    """The 256-cloud batch (as measure_batched) differentiable: one batched
    forward (VOX_FLAG_DIFFERENTIABLE) plus one batched adjoint with upstream
    dL/dvoxel ~ N(0, 1), against the batched forward alone."""
    from nanovdb_editor import workloads as W
    from nanovdb_editor.vox import FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS

    clouds, start, vs = W.batch_clouds(BATCHED["clouds"], 3 + rank, BATCHED["min_n"], BATCHED["max_n"])
    raw = W.concat(clouds).raw_arrays()
    dev = [torch.from_numpy(a).cuda() for a in raw[:5]]
    ins = (dev[0], dev[2], dev[3], dev[1], dev[4])
    out = {k: torch.empty_like(t) for k, t in zip(("means", "quats", "scales", "opacities", "colors"), ins)}
    flags = FLAG_RAW_INPUTS | FLAG_DIFFERENTIABLE
    _, _, voff = ctx.voxelize_batch(*ins, start, vs, 0.05, flags)
    vc = int(voff[-1])
    gen = torch.Generator(device="cuda").manual_seed(9)
    gd = torch.randn(vc, device="cuda", generator=gen)
    gc = torch.randn((vc, 3), device="cuda", generator=gen)
    torch.cuda.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(warmup):
            fn()
        res = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0.record(ext)
            fn()
            e1.record(ext)
            e1.synchronize()
            res.append(e0.elapsed_time(e1))
        return float(np.mean(res))

    fwd_ms = timed(lambda: ctx.voxelize_batch(*ins, start, vs, 0.05, FLAG_RAW_INPUTS))

    def fwd_bwd():
        ctx.voxelize_batch(*ins, start, vs, 0.05, flags)
        ctx.backward(*ins, gd, gc, out)

    fb_ms = timed(fwd_bwd)
    G = int(start[-1])
    return {"workload": "batched_fwd_bwd_256_clouds_1k-200k_vs0.002-0.02", "clouds": len(clouds), "gaussians": G,
            "batched_forward_ms": fwd_ms, "batched_fwd_bwd_ms": fb_ms, "fwd_bwd_over_forward": fb_ms / fwd_ms,
            "fwd_bwd_gaussians_per_s": G / (fb_ms * 1e-3),
            "parity": "batched adjoint = per-cloud adjoints (tests/test_gpu_batch.py); 1e-5 of each family's max vs FP64 "
                      "(tests/test_gpu_adjoint.py)"}


FIT = {"workload": "fit_500k_clusters64_vs0.004_200steps", "gaussians": 500_000, "clusters": 64, "voxel_size": 0.004,
       "steps": 200}


def measure_fit(ctx, torch, rank):
    """L2 fit (200 Adam steps, FP32) of 500K Gaussians (cluster distribution,
    voxel 0.004) to the grid of an independently seeded 500K set: forward,
    loss over the union of both grids' voxels, adjoint and update per step,
    CUDA events around each step."""
    from nanovdb_editor import workloads as W
    from nanovdb_editor.autograd import TargetGrid, l2_to_target, voxelize

    G, vs = FIT["gaussians"], FIT["voxel_size"]
    names = ("means", "quats", "scales", "opacities", "colors")

    def dev_params(seed):
        r = W.cluster_cloud(G, seed, clusters=FIT["clusters"]).raw_arrays()
        return {k: torch.from_numpy(a).cuda() for k, a in zip(names, (r[0], r[2], r[3], r[1], r[4]))}

    tgt = dev_params(201 + rank)
    tdens, _, _ = voxelize(*[tgt[k] for k in names], vs, raw=True, context=ctx)
    target = TargetGrid.from_last(ctx, tdens)
    leaves = {k: t.clone().requires_grad_(True) for k, t in dev_params(202 + rank).items()}
    lr = {"means": 2e-4, "quats": 1e-3, "scales": 2e-3, "opacities": 1e-2, "colors": 1e-2}
    opt = torch.optim.Adam([{"params": [leaves[k]], "lr": lr[k]} for k in names])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times, losses = [], []
    for _ in range(FIT["steps"]):
        torch.cuda.synchronize()
        e0.record()
        opt.zero_grad()
        density, _, _ = voxelize(*[leaves[k] for k in names], vs, raw=True, context=ctx)
        loss = l2_to_target(density, ctx, target)
        loss.backward()
        opt.step()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        losses.append(float(loss.detach()))
    ms = float(np.median(times))
    return {"workload": FIT["workload"], "gaussians": G, "steps": FIT["steps"], "ms_per_step": ms,
            "total_s": float(np.sum(times)) * 1e-3, "gaussians_per_s": G / (ms * 1e-3),
            "loss_first": losses[0], "loss_last": losses[-1], "loss_ratio": losses[-1] / losses[0],
            "note": "step = differentiable forward + L2 loss + adjoint + torch Adam (FP32); gradients checked against "
                    "FP64 finite differences and the FP64 adjoint in tests/test_oracle_adjoint.py, tests/test_gpu_adjoint.py"}


FIT_BF16 = {"workload": "fit_bf16_64_clouds_50k-1M_vs0.002-0.01_100steps", "clouds": 64, "min_n": 50_000,
            "max_n": 1_000_000, "vs_min": 0.002, "vs_max": 0.01, "steps": 100}


class _DeviceBytes:
    """A device pointer as a uint8 CUDA array (no copy)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


def measure_fit_bf16(ctx, torch, rank, steps=None):
    """Batched fitting loop: 64 clouds (log-uniform 50K-1M Gaussians, 1-16
    clusters of the 2M workload's distribution, voxel sizes log-uniform in
    [0.002, 0.01]) fitted to per-cloud target grids (independently seeded
    clouds of the same sizes and voxel sizes).  Attributes stored in bfloat16
    (VOX_FLAG_BF16_INPUTS), FP32 master copies and moments; per step one
    batched differentiable forward, the L2 loss per cloud, one batched
    adjoint (FP32 gradients) and the fused vox_adam_bf16 update.  At the end
    the smallest cloud's density and gradients are compared with the FP64
    oracle on the same (bfloat16) values."""
    import oracle as oracle_py
    from nanovdb_editor import workloads as W
    from nanovdb_editor.autograd import BatchTargetGrid, batch_voxel_keys, l2_to_batch_target
    from nanovdb_editor.grid import HEADER_DTYPE
    from nanovdb_editor.vox import FLAG_BF16_INPUTS, FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS

    F = FIT_BF16
    steps = steps or F["steps"]
    names = ("means", "quats", "scales", "opacities", "colors")
    clouds, start, vs = W.batch_clouds(F["clouds"], 301 + rank, F["min_n"], F["max_n"], vs_min=F["vs_min"], vs_max=F["vs_max"])
    targets = [W.cluster_cloud(c.n, 5000 + 97 * b + rank, clusters=1 + b % 16) for b, c in enumerate(clouds)]
    G = int(start[-1])
    flags = FLAG_RAW_INPUTS | FLAG_DIFFERENTIABLE | FLAG_BF16_INPUTS

    def as_params(cl):
        r = W.concat(cl).raw_arrays()
        return {k: torch.from_numpy(a).cuda() for k, a in zip(names, (r[0], r[2], r[3], r[1], r[4]))}

    def density_of(ptr, goff):
        """the batch's density channel, value index order (clouds back to back)"""
        buf = torch.as_tensor(_DeviceBytes(ptr, int(goff[-1])), device="cuda")
        heads = np.frombuffer(torch.stack([buf[int(o): int(o) + 256] for o in goff[:-1]]).cpu().numpy().tobytes(),
                              HEADER_DTYPE)
        parts = [buf[int(o) + int(h["density_offset"]): int(o) + int(h["density_offset"]) + 4 * int(h["value_count"])]
                 for o, h in zip(goff[:-1], heads)]
        return torch.cat(parts).view(torch.float32)

    tp = {k: v.to(torch.bfloat16).contiguous() for k, v in as_params(targets).items()}
    torch.cuda.synchronize()
    ptr, goff, voff = ctx.voxelize_batch(*[tp[k] for k in names], start, vs, 0.05, flags)
    tkeys, tvalid = batch_voxel_keys(ctx, voff, "cuda")
    target = BatchTargetGrid(tkeys, tvalid, density_of(ptr, goff).clone())
    del tp
    master = as_params(clouds)
    bf = {k: v.to(torch.bfloat16).contiguous() for k, v in master.items()}
    mom = {k: (torch.zeros_like(v), torch.zeros_like(v)) for k, v in master.items()}
    grads = {k: torch.empty_like(v) for k, v in master.items()}
    lr = {"means": 2e-4, "quats": 1e-3, "scales": 2e-3, "opacities": 1e-2, "colors": 1e-2}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ext = torch.cuda.ExternalStream(ctx.stream)
    times, losses = [], []
    pairs = voxels = 0
    for t in range(1, steps + 1):
        torch.cuda.synchronize()
        e0.record(ext)
        ptr, goff, voff = ctx.voxelize_batch(*[bf[k] for k in names], start, vs, 0.05, flags)
        st = ctx.stats()
        pairs, voxels = int(st["pairs"]), int(st["voxels"])
        density = density_of(ptr, goff)
        keys, valid = batch_voxel_keys(ctx, voff, "cuda")
        loss, gd = l2_to_batch_target(density, keys, valid, target)
        torch.cuda.synchronize()
        ctx.backward(*[bf[k] for k in names], gd.contiguous(), None, grads)
        if t == steps:  # the values this step's density and gradients belong to, before the update
            b = int(np.argmin([c.n for c in clouds]))
            g0, g1 = int(start[b]), int(start[b + 1])
            cur = {k: bf[k][g0:g1].to(torch.float32).cpu().numpy() for k in names}
        for k in names:
            ctx.adam_bf16(master[k], mom[k][0], mom[k][1], grads[k], bf[k], t, lr[k])
        e1.record(ext)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        losses.append(loss)
    # FP64 check on the smallest cloud: the last step's density and gradients
    v0, v1 = int(voff[b]), int(voff[b + 1])
    act = oracle_py.preprocess([cur["means"], cur["opacities"], cur["quats"], cur["scales"], cur["colors"]])
    ref = oracle_py.OracleResult(act, float(vs[b]), 0.05, window_mode=oracle_py.OV_MODE_SMOOTH)
    vals = ref.values()
    d64 = vals["density64"]
    dens_err = float(np.abs(density[v0:v1].cpu().numpy().astype(np.float64) - d64).max()) / float(np.abs(d64).max())
    an = ref.smooth_grad64(cur, True, gd[v0:v1].cpu().numpy().astype(np.float64), None)
    grad_err = {}
    for k in names:
        got = grads[k][g0:g1].cpu().numpy().astype(np.float64).reshape(an[k].shape)
        grad_err[k] = float(np.abs(got - an[k]).max()) / max(float(np.abs(an[k]).max()), 1e-30)
    ref.close()
    ms = float(np.median(times))
    return {"workload": F["workload"], "clouds": len(clouds), "gaussians": G, "steps": steps, "pairs": pairs,
            "voxels": voxels, "ms_per_step": ms, "total_s": float(np.sum(times)) * 1e-3,
            "gaussians_per_s": G / (ms * 1e-3), "loss_first": losses[0], "loss_last": losses[-1],
            "storage": "bfloat16 attributes, FP32 masters / moments / gradients / accumulation",
            "fp64_check": {"cloud": b, "gaussians": g1 - g0, "density_rel_err": dens_err, "grad_rel_err": grad_err,
                           "tolerance": 1e-5}}


VOXELBVH = {"workload": "voxelbvh_ijkl_2M_clusters64_res512", "gaussians": 2_000_000, "clusters": 64, "resolution": 512}
VOXELBVH_METRIC = "Gaussians/s ingested into VoxelBVH keys (ijkl_from_gaussians)"


def measure_voxelbvh_form(ctx, torch, rank, steps, warmup, flush):
    """VoxelBVH Gaussian ingestion on the main cloud's distribution (2M
    Gaussians, 64 clusters, resolution 512), activated inputs resident in HBM,
    CUDA events on the library's stream; `python bench.py --workload
    voxelbvh` prints the full line for it (e2e, roofline, CPU baseline)."""
    from nanovdb_editor import workloads as W

    cloud = W.cluster_cloud(VOXELBVH["gaussians"], 1 + rank, clusters=VOXELBVH["clusters"])
    dev = [torch.from_numpy(np.ascontiguousarray(cloud[k], dtype=np.float32)).cuda()
           for k in ("means", "opacities", "quats", "scales")]
    res = VOXELBVH["resolution"]
    ext = torch.cuda.ExternalStream(ctx.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(warmup):
        out = ctx.voxelbvh_ijkl_from_gaussians(*dev, res)
    times, stats = [], []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record(ext)
        out = ctx.voxelbvh_ijkl_from_gaussians(*dev, res)
        ev1.record(ext)
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
        stats.append(ctx.stats())
    ms = float(np.mean(times))
    return {
        "workload": VOXELBVH["workload"],
        "gaussians": VOXELBVH["gaussians"],
        "ms_per_call": ms,
        "gaussians_per_s": VOXELBVH["gaussians"] / (ms * 1e-3),
        "stages_ms": {k: float(np.mean([x[f"ms_vb_{k}"] for x in stats])) for k in ("keys", "sort", "ranges")},
        "ranges": int(out["range_count"]),
        "sort_bits": int(stats[-1]["vb_sort_bits"]),
        "parity": "keys, ids, range headers and world box bit-exact to the oracle (tests/test_gpu_voxelbvh.py)",
    }


def voxelbvh_cpu(target_s=10.0):
    """The oracle's VoxelBVH ingestion on a bounded sample, all host cores
    (per-Gaussian work split over threads; the key sort is serial)."""
    import oracle as oracle_py
    from nanovdb_editor import workloads as W

    oracle_py.build()
    cores = os.cpu_count() or 1
    n, rate, sample = 100_000, None, None
    for _ in range(3):
        cloud = W.cluster_cloud(n, 1, clusters=max(1, int(64 * n / VOXELBVH["gaussians"])))
        t0 = time.perf_counter()
        out = oracle_py.voxelbvh_ijkl(cloud, VOXELBVH["resolution"], nthreads=cores)
        dt = time.perf_counter() - t0
        rate = n / dt if out["ranges"] > 0 else None
        sample = f"{n} Gaussians of the 2M-cluster distribution, resolution {VOXELBVH['resolution']}, {dt:.1f}s, {cores} threads"
        if dt > target_s / 3 or n >= VOXELBVH["gaussians"]:
            break
        n = int(min(VOXELBVH["gaussians"], n * max(2.0, target_s / max(dt, 1e-3) / 2)))
    return {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}


def run_voxelbvh(args, rank, world, local):
    """VoxelBVH Gaussian ingestion (ijkl_from_gaussians): one step = world box,
    level search, 8 keys per Gaussian, key sort and range headers for one
    cloud; inputs resident in HBM, L2 flushed between steps."""
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    from nanovdb_editor import replicas as R
    from nanovdb_editor import workloads as W
    from nanovdb_editor.vox import VoxContext

    G, res = args.gaussians, VOXELBVH["resolution"]
    cloud = W.cluster_cloud(G, 1 + rank, clusters=64)
    host = [np.ascontiguousarray(cloud[k], dtype=np.float32) for k in ("means", "opacities", "quats", "scales")]
    dev = [torch.from_numpy(a).cuda() for a in host]
    ctx = VoxContext(local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ext = torch.cuda.ExternalStream(ctx.stream)
    for _ in range(args.warmup):
        out = ctx.voxelbvh_ijkl_from_gaussians(*dev, res)
    torch.cuda.synchronize()
    times, stats = [], []
    if dist:
        dist.barrier()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            start.record(ext)
            out = ctx.voxelbvh_ijkl_from_gaussians(*dev, res)
            end.record(ext)
            end.synchronize()
            times.append(start.elapsed_time(end))
            stats.append(ctx.stats())
    if dist:
        dist.barrier()
    ms = R.max_over_ranks(sum(times) / len(times), dist, device="cuda")
    value = R.job_rate(world * G, ms)
    ranges = out["range_count"]

    # e2e: pinned host inputs copied in and all outputs read back every step
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(a).pin_memory() for a in host]
        outs = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in out.items() if hasattr(v, "shape")}
        h2d = sum(int(t.numel()) * 4 for t in pinned)
        d2h = sum(int(t.numel()) * t.element_size() for t in outs.values())
        e2e_t = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d = [t.cuda(non_blocking=True) for t in pinned]
            o = ctx.voxelbvh_ijkl_from_gaussians(*d, res)
            for k in outs:
                outs[k].copy_(o[k], non_blocking=True)
            torch.cuda.synchronize()
            e2e_t.append(time.perf_counter() - t0)
        e2e_s = R.max_over_ranks(sum(e2e_t) / len(e2e_t), dist, device="cuda")
        e2e = {"value": R.job_rate(world * G, e2e_s * 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3}

    st = stats[-1]
    N = 8 * G
    bits = int(st["vb_sort_bits"])
    kb = 4 if bits <= 32 else 8
    passes = (bits + 7) // 8
    stage_ms = {k: float(np.mean([x[f"ms_vb_{k}"] for x in stats])) for k in ("keys", "sort", "ranges")}
    # algorithmic bytes per stage
    stage_bytes = {
        "keys": G * 44 * 2 + N * 12,  # attributes read by the box and key kernels, keys + ids out
        "sort": N * (8 + kb) + N * kb + passes * 2 * N * (kb + 4),  # compress, histogram, passes (key + id)
        "ranges": N * kb * 2 + N * 8 + N * 8 + N * 8,  # two key reads, headers, 64-bit keys, ids
    }
    peak, peak_kind = load_peaks()
    sort_gbs = stage_bytes["sort"] / (stage_ms["sort"] * 1e-3) / 1e9
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    cpu = voxelbvh_cpu() if rank == 0 and not args.no_cpu_baseline and world == 1 else None
    if rank == 0:
        line = {
            "metric": VOXELBVH_METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": dict(VOXELBVH, gaussians=G, parallelism=f"replicas{world}" if world > 1 else "single",
                           l2="256 MB flush between steps", inputs="activated (means, opacities, quats wxyz, scales)"),
            "e2e": e2e,
            "gpu_launches": int(sum(x["vb_launches"] for x in stats)),
            "roofline": {
                "bound": "hbm",
                "kernel": "sort",
                "achieved": sort_gbs,
                "peak": peak,
                "unit": "GB/s",
                "frac": sort_gbs / peak,
                "traffic": None,
                "peak_source": peak_kind,
                "algorithmic_bytes": stage_bytes["sort"],
                "basis": f"key sort of {N} slots: compression (8 B in, {kb} B out), histogram read, {passes} onesweep passes of {kb}+4 B read and written ({bits}-bit compressed keys)",
                "dominant_stage": dom,
                "stages_gbs": {k: stage_bytes[k] / (stage_ms[k] * 1e-3) / 1e9 for k in stage_ms},
            },
            "stages_ms": stage_ms,
            "counts": {"slots": N, "ranges": ranges, "sort_bits": bits},
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload == "voxelbvh":
        res = [voxelbvh_cpu() for _ in range(max(1, args.steps))]
        vals = [r["value"] for r in res if r["value"]]
        v = statistics.median(vals) if vals else None
        line = {
            "impl": "reference",
            "metric": VOXELBVH_METRIC,
            "value": v,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": dict(VOXELBVH, note="CPU restatement of the reference's VoxelBVH ingestion (its path runs only on Vulkan)"),
            "cpu_baseline": {"kind": "port", "cores": res[-1]["cores"], "sample": res[-1]["sample"], "value": v, "unit": UNIT},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    res = []
    for _ in range(max(1, args.steps)):
        res.append(cpu_baseline())
    vals = [r["value"] for r in res if r["value"]]
    v = statistics.median(vals) if vals else None
    cfg0 = cpu_cfg0()
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": run_config(args.gaussians, world),
        "cpu_baseline": {"kind": "port", "cores": res[-1]["cores"], "sample": res[-1]["sample"], "value": v, "unit": UNIT,
                         "implementation": "CPU restatement of the reference path (oracle/vox_oracle.c); the reference's "
                                           "own path runs only on Vulkan, which this box cannot bring up",
                         "pairs_per_s": statistics.median([r["pairs_per_s"] for r in res if r["pairs_per_s"]] or [0]),
                         "voxels_per_s": statistics.median([r["voxels_per_s"] for r in res if r["voxels_per_s"]] or [0])},
        "cfg0_full": cfg0,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--gaussians", type=int, default=WORKLOAD["gaussians"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer C-ABI measurement (profiling runs)")
    ap.add_argument("--no-forms", action="store_true", help="skip the forward+backward and batched forms")
    ap.add_argument("--workload", default="voxelize", choices=["voxelize", "voxelbvh"],
                    help="voxelbvh: VoxelBVH Gaussian ingestion (ijkl_from_gaussians) instead of node2 voxelization")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "voxelbvh":
        run_voxelbvh(args, rank, world, local)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    from ctypes import POINTER, byref, c_float, c_uint32, pointer

    from nanovdb_editor import replicas as R
    from nanovdb_editor import workloads as W
    from nanovdb_editor.compute import Compute, pnanovdb_ComputeArray
    from nanovdb_editor.raster import Raster
    from nanovdb_editor.vox import FLAG_RAW_INPUTS, VoxContext

    G = args.gaussians
    vs = WORKLOAD["voxel_size"]
    cloud = W.cluster_cloud(G, 1 + rank, clusters=64)
    raw = cloud.raw_arrays()  # [means, logit, quats, log_s, sh0, sh_n]
    dev = [torch.from_numpy(a).cuda() for a in raw[:5]]
    ctx = VoxContext(local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    ext_stream = torch.cuda.ExternalStream(ctx.stream)

    def step():
        # inputs resident in HBM: means, quats, log scales, logits, SH0
        ctx.voxelize(dev[0], dev[2], dev[3], dev[1], dev[4], vs, 0.05, FLAG_RAW_INPUTS)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    times, stats = [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            start.record(ext_stream)
            step()
            end.record(ext_stream)
            end.synchronize()
            times.append(start.elapsed_time(end))
            stats.append(ctx.stats())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = R.max_over_ranks(sum(times) / len(times), dist, device="cuda")
    value = R.job_rate(world * G, ms)

    # the same step in the reference's node order (its window-by-window build), device-timed
    from nanovdb_editor.vox import FLAG_WINDOW_ORDER

    def step_window():
        ctx.voxelize(dev[0], dev[2], dev[3], dev[1], dev[4], vs, 0.05, FLAG_RAW_INPUTS | FLAG_WINDOW_ORDER)

    step_window()
    wtimes = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        start.record(ext_stream)
        step_window()
        end.record(ext_stream)
        end.synchronize()
        wtimes.append(start.elapsed_time(end))
    w_ms = R.max_over_ranks(sum(wtimes) / len(wtimes), dist, device="cuda")
    window_order = {"ms_per_step": w_ms, "value": R.job_rate(world * G, w_ms), "unit": UNIT,
                    "note": "the same step with VOX_FLAG_WINDOW_ORDER: node2 bytes in the reference's node order"}

    # ---- e2e through the reference-facing C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        comp = Compute(device_index=local)
        raster = Raster(comp)
        pinned = [torch.from_numpy(a).pin_memory() for a in raw]
        arrays = []
        for t in pinned:
            arr = pnanovdb_ComputeArray()
            arr.data = t.data_ptr()
            arr.element_size = 4
            arr.element_count = t.numel()
            arrays.append(arr)
        h2d = sum(int(t.numel()) * 4 for t in pinned[:5])
        out = raster.raster_to_nanovdb_from_arrays(vs, arrays)  # warm
        comp.destroy_array(out)
        e2e_times, d2h = [], 0
        if dist:
            dist.barrier()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = raster.raster_to_nanovdb_from_arrays(vs, arrays)
            e2e_times.append(time.perf_counter() - t0)
            d2h = int(out.element_size * out.element_count)
            comp.destroy_array(out)
        e2e_s = R.max_over_ranks(sum(e2e_times) / len(e2e_times), dist, device="cuda")
        e2e_value = R.job_rate(world * G, e2e_s * 1e3)
        e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3}

    # ---- roofline of the dominant stage
    st = stats[-1]
    P = st["pairs"]
    Q = st["leaf_pairs"]
    NCL = st["candidate_leaves"]
    V = st["voxels"]
    passes = st["sort_passes"]
    A = 56
    # algorithmic bytes per stage: what each stage must read and write once
    stage_bytes = {
        "prep": G * (A + 128 + 8),  # raw attributes in, record + footprint out
        "leaf_pairs": 2 * G * 128 + 12 * Q,  # records read by the count and write passes, (key, index, id) out
        "sort": Q * (4 + 16 * passes),  # histogram read + per pass read/write (key, value)
        "leaf_walk": 8 * Q + 128 * Q + 72 * NCL + 24 * V,  # pair lists, record gathers, masks, staged values
        "tree_values": 60 * V,  # voxel keys, runs, node tables, values
    }
    stage_ms = {
        "prep": float(np.mean([s["ms_prep"] for s in stats])),
        "leaf_pairs": float(np.mean([s["ms_emit"] for s in stats])),
        "sort": float(np.mean([s["ms_sort"] for s in stats])),
        "leaf_walk": float(np.mean([s["ms_accumulate"] for s in stats])),
        "tree_values": float(np.mean([s["ms_build"] for s in stats])),
    }
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    peak, peak_kind = load_peaks()
    # algorithmic bytes of the pair work: emit (8 B key + 4 B id), one 8-bit
    # onesweep pass per 8 varying key bits (read + write key and id), one read
    # of the sorted pairs to accumulate, density + colour + RGBA8 per voxel
    sort_passes_pairs = (st["key_bits"] + 7) // 8
    pair_bytes = 12 * P + 24 * P * sort_passes_pairs + 12 * P + 20 * V
    topo_bytes = 80 * st["leaves"] + 1100 * st["lowers"] + 8300 * st["uppers"]
    step_bytes = 2 * G * A + pair_bytes + topo_bytes
    achieved = pair_bytes / (stage_ms["leaf_walk"] * 1e-3) / 1e9
    step_achieved = step_bytes / (ms * 1e-3) / 1e9
    own_achieved = stage_bytes[dom] / (stage_ms[dom] * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        # DRAM bytes ncu measured per launch of the dominant kernel, scaled to this workload
        t = json.load(open(tp)).get(dom)
        if t and t.get("voxels"):
            traffic = t["bytes"] * V / t["voxels"]

    forms = {}
    if not args.no_forms:
        forms["fwd_bwd"] = measure_fwd_bwd(ctx, torch, rank, args.steps, args.warmup, flush)
        forms["batched"] = measure_batched(ctx, torch, rank, args.steps, args.warmup, flush)
        for name, fn in (("batched_fwd_bwd", lambda: measure_batched_fwd_bwd(ctx, torch, rank, args.steps, args.warmup, flush)),
                         ("fit", lambda: measure_fit(ctx, torch, rank)),
                         ("fit_bf16", lambda: measure_fit_bf16(ctx, torch, rank))):
            try:
                forms[name] = fn()
            except Exception as e:  # a secondary row: never lose the main line to it
                forms[name] = {"error": f"{type(e).__name__}: {e}"}
        try:
            forms["voxelbvh"] = measure_voxelbvh_form(ctx, torch, rank, args.steps, args.warmup, flush)
        except Exception as e:  # a secondary row: never lose the main line to it
            forms["voxelbvh"] = {"error": f"{type(e).__name__}: {e}"}

    cfg0 = None
    if not args.no_forms:
        cfg0 = {"gpu": gpu_cfg0(ctx, torch, args.steps, args.warmup, flush)}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cpu = cpu_baseline()
        if cfg0 is not None:
            cfg0["cpu"] = cpu_cfg0()
            cfg0["gpu_over_cpu"] = cfg0["gpu"]["gaussians_per_s"] / cfg0["cpu"]["gaussians_per_s"]

    if rank == 0:
        clk = clocks.summary()
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": run_config(G, world),
            "window_order": window_order,
            "cfg0_full": cfg0,
            "e2e": e2e,
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "roofline": {
                "bound": "hbm",
                "kernel": "leaf_walk",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": traffic,
                "peak_source": peak_kind,
                "algorithmic_bytes": pair_bytes,
                "basis": f"pair work the leaf walk performs: 12 B/pair emit + 24 B/pair x {sort_passes_pairs} sort passes ({st['key_bits']}-bit voxel keys) + 12 B/pair accumulate + 20 B/voxel values",
                "step": {"achieved": step_achieved, "frac": step_achieved / peak, "bytes": step_bytes},
                "own_bytes": {"bytes": stage_bytes[dom], "achieved": own_achieved, "frac": own_achieved / peak,
                              "note": "the leaf walk's own reads and writes: it never materialises the pairs, so DRAM stays far below peak; it is FP32/FP64 instruction-issue bound"},
            },
            "stages_ms": stage_ms,
            "counts": {k: st[k] for k in ("candidates", "pairs", "voxels", "uppers", "lowers", "leaves", "key_bits", "sort_passes", "sort_shape", "leaf_pairs", "candidate_leaves")},
            "pairs_per_s": world * P / (ms * 1e-3),
            "voxels_per_s": world * st["voxels"] / (ms * 1e-3),
            "clocks": clk,
            "forms": forms,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
