"""GPU parity of the differentiable path.

Forward: the differentiable channels of the CUDA path are bit-identical to
the oracle's float restatement (same per-pair arithmetic, exact fixed-point
sums) and within 1e-5 of the channel maximum against FP64.
Backward: the CUDA adjoint (vox_backward) is within 1e-5 of each parameter
family's maximum against the oracle's FP64 adjoint, which
tests/test_oracle_adjoint.py pins with FP64 central differences.
"""

import numpy as np
import pytest

from nanovdb_editor import workloads as W
from test_oracle_adjoint import FAMILIES, raw_params, smooth_forward, upstream

pytestmark = pytest.mark.gpu

REL = 1e-5
NAMES = ("means", "quats", "scales", "opacities", "colors")


def _dev(params):
    import torch

    return {k: torch.from_numpy(np.ascontiguousarray(params[k])).cuda() for k in NAMES}


def _flags():
    from nanovdb_editor.vox import FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS

    return FLAG_DIFFERENTIABLE | FLAG_RAW_INPUTS


@pytest.mark.parametrize("n,seed,vs", [(20_000, 41, 0.004), (3000, 42, 0.002)])
def test_smooth_forward_parity(vox_ctx, oracle_mod, n, seed, vs):
    params = raw_params(W.cluster_cloud(n, seed, clusters=8), seed)
    g = vox_ctx.voxelize_host(*[params[k] for k in NAMES], vs, 0.05, flags=_flags())
    ref = smooth_forward(oracle_mod, params, vs)
    assert ref.counts["error"] == 0 and ref.counts["V"] > 0
    k_ref, i_ref = ref.pairs()
    k_got, i_got = vox_ctx.pairs()
    np.testing.assert_array_equal(k_got, k_ref)
    np.testing.assert_array_equal(i_got, i_ref)
    assert np.array_equal(g.node2, ref.node2())
    v = ref.values()
    np.testing.assert_array_equal(g.rgba8, v["rgba8"])
    np.testing.assert_array_equal(g.density, v["density"])
    np.testing.assert_array_equal(g.color, v["color"])
    dmax = float(np.abs(v["density64"]).max())
    assert float(np.abs(g.density - v["density64"]).max()) <= REL * dmax
    cmax = float(np.abs(v["color64"]).max())
    assert float(np.abs(g.color - v["color64"]).max()) <= REL * cmax
    ref.close()


def _gpu_grads(vox_ctx, dev, vs, gd, gc):
    import torch

    vox_ctx.voxelize(*[dev[k] for k in NAMES], vs, 0.05, flags=_flags())
    vc = int(vox_ctx.stats()["value_count"])
    assert vc == gd.shape[0]
    out = {k: torch.empty_like(dev[k]) for k in NAMES}
    vox_ctx.backward(*[dev[k] for k in NAMES], torch.from_numpy(gd).cuda(), torch.from_numpy(gc).cuda(), out)
    return {k: out[k].cpu().numpy().astype(np.float64) for k in NAMES}


@pytest.mark.parametrize("n,seed,vs", [(20_000, 43, 0.004), (100_000, 44, 0.004)])
def test_backward_matches_fp64_adjoint(vox_ctx, oracle_mod, n, seed, vs):
    params = raw_params(W.cluster_cloud(n, seed, clusters=16), seed)
    ref = smooth_forward(oracle_mod, params, vs)
    gd64, gc64 = upstream(ref.counts["value_count"], seed + 100)
    gd, gc = gd64.astype(np.float32), gc64.astype(np.float32)
    got = _gpu_grads(vox_ctx, _dev(params), vs, gd, gc)
    an = ref.smooth_grad64(params, True, gd.astype(np.float64), gc.astype(np.float64))
    for k in NAMES:
        scale = float(np.abs(an[k]).max())
        err = float(np.abs(got[k].reshape(an[k].shape) - an[k]).max())
        assert scale > 0 and err <= REL * scale, (k, err, scale)
    ref.close()


def test_backward_density_only_and_no_upstream(vox_ctx, oracle_mod):
    import torch

    params = raw_params(W.cluster_cloud(5000, 45, clusters=4), 45)
    ref = smooth_forward(oracle_mod, params, 0.004)
    gd64, _ = upstream(ref.counts["value_count"], 145)
    gd = gd64.astype(np.float32)
    dev = _dev(params)
    vox_ctx.voxelize(*[dev[k] for k in NAMES], 0.004, 0.05, flags=_flags())
    out = {k: torch.empty_like(dev[k]) for k in NAMES}
    vox_ctx.backward(*[dev[k] for k in NAMES], torch.from_numpy(gd).cuda(), None, out)
    an = ref.smooth_grad64(params, True, gd.astype(np.float64), None)
    for k in NAMES:
        scale = float(np.abs(an[k]).max())
        err = float(np.abs(out[k].cpu().numpy().reshape(an[k].shape) - an[k]).max())
        assert err <= REL * max(scale, 1e-30), (k, err, scale)
    assert float(np.abs(out["colors"].cpu().numpy()).max()) == 0.0  # colour gradients need dL/d colour
    vox_ctx.backward(*[dev[k] for k in NAMES], None, None, out)
    for k in NAMES:
        assert float(out[k].abs().max()) == 0.0
    ref.close()


def test_backward_requires_differentiable_forward(vox_ctx):
    from nanovdb_editor.exceptions import PipelineError
    import torch

    params = raw_params(W.cluster_cloud(2000, 46, clusters=2), 46)
    dev = _dev(params)
    vox_ctx.voxelize(*[dev[k] for k in NAMES], 0.004, 0.05, flags=1)
    out = {k: torch.empty_like(dev[k]) for k in NAMES}
    with pytest.raises(PipelineError):
        vox_ctx.backward(*[dev[k] for k in NAMES], None, None, out)


def test_autograd_function(vox_ctx, oracle_mod):
    import torch

    from nanovdb_editor.autograd import voxelize
    from nanovdb_editor.exceptions import PipelineError

    params = raw_params(W.cluster_cloud(20_000, 47, clusters=8), 47)
    dev = _dev(params)
    leaves = {k: dev[k].clone().requires_grad_(True) for k in NAMES}
    density, color, grid = voxelize(*[leaves[k] for k in NAMES], 0.004, raw=True, context=vox_ctx)
    vc = density.shape[0]
    gd64, gc64 = upstream(vc, 147)
    gd = torch.from_numpy(gd64.astype(np.float32)).cuda()
    gc = torch.from_numpy(gc64.astype(np.float32)).cuda()
    loss = (density * gd).sum() + (color * gc).sum()
    loss.backward()
    ref = smooth_forward(oracle_mod, params, 0.004)
    an = ref.smooth_grad64(params, True, gd.cpu().numpy().astype(np.float64), gc.cpu().numpy().astype(np.float64))
    for k in NAMES:
        scale = float(np.abs(an[k]).max())
        err = float(np.abs(leaves[k].grad.cpu().numpy().astype(np.float64).reshape(an[k].shape) - an[k]).max())
        assert err <= REL * scale, (k, err, scale)
    ref.close()
    # a later forward on the same context invalidates the earlier graph
    d1, _, _ = voxelize(*[leaves[k] for k in NAMES], 0.004, raw=True, context=vox_ctx)
    d2, _, _ = voxelize(*[leaves[k] for k in NAMES], 0.004, raw=True, context=vox_ctx)
    with pytest.raises(PipelineError):
        d1.sum().backward()


def test_fit_loop_reduces_l2(vox_ctx):
    """A short L2 fit (Adam) of perturbed Gaussians to the grid of the originals."""
    import torch

    from nanovdb_editor.autograd import TargetGrid, l2_to_target, voxelize

    vs = 0.004
    params = raw_params(W.cluster_cloud(20_000, 48, clusters=4), 48)
    dev = _dev(params)
    tdens, _, _ = voxelize(*[dev[k] for k in NAMES], vs, raw=True, context=vox_ctx)
    target = TargetGrid.from_last(vox_ctx, tdens)
    g = torch.Generator(device="cuda").manual_seed(0)
    init = dict(dev)
    init["means"] = dev["means"] + 0.002 * torch.randn(dev["means"].shape, device="cuda", generator=g)
    init["scales"] = dev["scales"] + 0.3 * torch.randn(dev["scales"].shape, device="cuda", generator=g)
    init["opacities"] = dev["opacities"] - 0.5
    leaves = {k: init[k].clone().requires_grad_(True) for k in NAMES}
    opt = torch.optim.Adam(list(leaves.values()), lr=2e-3)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        density, _, _ = voxelize(*[leaves[k] for k in NAMES], vs, raw=True, context=vox_ctx)
        loss = l2_to_target(density, vox_ctx, target)
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    assert all(np.isfinite(losses))
    assert losses[-1] < 0.7 * losses[0], losses
