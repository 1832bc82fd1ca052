"""Batched voxelization: many clouds of uneven size and voxel size in one call.

Every cloud's grid in the batched output must be byte-identical to the grid
the single-cloud call produces for that cloud alone (header, node2 region,
bbox, RGBA8, density, colour), and one cloud is also checked against the
oracle directly.  The differentiable batched call's adjoint equals the
per-cloud adjoints.
"""

import numpy as np
import pytest

from nanovdb_editor import workloads as W

pytestmark = pytest.mark.gpu

NAMES = ("means", "quats", "scales", "opacities", "colors")


def _batch(seed=5, count=12):
    clouds, start, vs = W.batch_clouds(count, seed, min_n=200, max_n=20_000, vs_min=0.002, vs_max=0.02)
    # an empty cloud and a cloud whose Gaussians are all below the opacity cutoff
    empty = W.cluster_cloud(0, 1, clusters=1)
    dim = W.cluster_cloud(300, 2, clusters=2)
    dim["opacities"][:] = 0.005
    clouds = clouds[:3] + [empty] + clouds[3:6] + [dim] + clouds[6:]
    vs = np.concatenate([vs[:3], [0.004], vs[3:6], [0.004], vs[6:]]).astype(np.float32)
    sizes = [c.n for c in clouds]
    start = np.zeros(len(clouds) + 1, np.int64)
    start[1:] = np.cumsum(sizes)
    return clouds, start, vs


def _dev(cloud):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(cloud[k])).cuda() for k in NAMES]


def test_batch_grids_equal_single_calls(vox_ctx, oracle_mod):
    clouds, start, vs = _batch()
    allc = W.concat(clouds)
    _, goff, voff = vox_ctx.voxelize_batch(*_dev(allc), start, vs)
    grids = vox_ctx.grids(goff)
    assert len(grids) == len(clouds)
    for b, (c, v) in enumerate(zip(clouds, vs)):
        single = vox_ctx.voxelize_host(*[c[k] for k in NAMES], float(v))
        assert np.array_equal(grids[b].buf, single.buf), f"cloud {b}: batched grid differs from the single-cloud grid"
        assert int(voff[b + 1] - voff[b]) == single.value_count
    # direct oracle anchor for one non-trivial cloud
    b = int(np.argmax([c.n for c in clouds]))
    ref = oracle_mod.OracleResult(clouds[b], float(vs[b]), 0.05, window_mode=0)
    assert np.array_equal(grids[b].node2, ref.node2())
    vals = ref.values()
    np.testing.assert_array_equal(grids[b].rgba8, vals["rgba8"])
    np.testing.assert_array_equal(grids[b].density, vals["density"])
    ref.close()


def test_batch_rejects_bad_layout(vox_ctx):
    from nanovdb_editor.exceptions import PipelineError

    clouds, start, vs = _batch(6, 4)
    allc = W.concat(clouds)
    bad = start.copy()
    bad[-1] -= 1
    with pytest.raises(PipelineError):
        vox_ctx.voxelize_batch(*_dev(allc), bad, vs)
    bad_vs = vs.copy()
    bad_vs[1] = 0.0
    with pytest.raises(PipelineError):
        vox_ctx.voxelize_batch(*_dev(allc), start, bad_vs)


def test_batch_backward_equals_per_cloud(vox_ctx):
    import torch

    from nanovdb_editor.vox import FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS

    flags = FLAG_DIFFERENTIABLE | FLAG_RAW_INPUTS
    clouds, start, vs = _batch(7, 6)
    raws = []
    for c in clouds:
        m, lg, q, ls, sh, _ = c.raw_arrays()
        raws.append({"means": m, "quats": q, "scales": ls, "opacities": lg, "colors": sh})
    allr = {k: np.ascontiguousarray(np.concatenate([r[k] for r in raws], axis=0)) for k in NAMES}
    dev = [torch.from_numpy(allr[k]).cuda() for k in NAMES]
    _, goff, voff = vox_ctx.voxelize_batch(*dev, start, vs, flags=flags)
    total = int(voff[-1])
    rng = np.random.default_rng(9)
    gd = rng.standard_normal(total).astype(np.float32)
    gc = rng.standard_normal((total, 3)).astype(np.float32)
    out = {k: torch.empty_like(t) for k, t in zip(NAMES, dev)}
    vox_ctx.backward(*dev, torch.from_numpy(gd).cuda(), torch.from_numpy(gc).cuda(), out)
    got = {k: out[k].cpu().numpy() for k in NAMES}
    for b, r in enumerate(raws):
        n = int(start[b + 1] - start[b])
        if n == 0:
            continue
        d1 = [torch.from_numpy(np.ascontiguousarray(r[k])).cuda() for k in NAMES]
        vox_ctx.voxelize(*d1, float(vs[b]), 0.05, flags)
        v0, v1 = int(voff[b]), int(voff[b + 1])
        o1 = {k: torch.empty_like(t) for k, t in zip(NAMES, d1)}
        vox_ctx.backward(*d1, torch.from_numpy(gd[v0:v1].copy()).cuda(), torch.from_numpy(gc[v0:v1].copy()).cuda(), o1)
        for k in NAMES:
            want = o1[k].cpu().numpy()
            have = got[k][int(start[b]) : int(start[b + 1])]
            scale = float(np.abs(want).max()) if want.size else 0.0
            assert float(np.abs(have - want).max(initial=0.0)) <= 1e-6 * max(scale, 1e-30), (b, k)
