"""BF16 attribute storage (VOX_FLAG_BF16_INPUTS) and the fused Adam step.

Attributes stored in bfloat16 are read exactly as float (a bfloat16 is the
upper half of a float), and everything after that is the FP32 / FP64
arithmetic of the float path.  So a BF16 call must equal, bit for bit, the
float call given the same values as float32 - grid, node2 region, every value
channel, and every gradient of the adjoint - and its error against FP64 is the
float path's: the gradients are checked against the oracle's FP64 adjoint
within 1e-5 of each family's maximum.  vox_adam_bf16 is checked against an
FP64 evaluation of the same Adam step.
"""

import numpy as np
import pytest

from nanovdb_editor import workloads as W
from test_oracle_adjoint import raw_params, smooth_forward, upstream

pytestmark = pytest.mark.gpu

REL = 1e-5
NAMES = ("means", "quats", "scales", "opacities", "colors")


def _pair(params):
    """(bfloat16 CUDA tensors, the same values as float32 CUDA tensors)"""
    import torch

    bf = {k: torch.from_numpy(np.ascontiguousarray(params[k])).to(torch.bfloat16).cuda() for k in NAMES}
    return bf, {k: v.to(torch.float32).contiguous() for k, v in bf.items()}


def test_bf16_forward_and_adjoint_equal_float_path(vox_ctx, oracle_mod):
    import torch

    from nanovdb_editor.vox import FLAG_BF16_INPUTS, FLAG_DIFFERENTIABLE, FLAG_RAW_INPUTS

    vs = 0.004
    params = raw_params(W.cluster_cloud(20_000, 61, clusters=8), 61)
    bf, f32 = _pair(params)
    flags = FLAG_DIFFERENTIABLE | FLAG_RAW_INPUTS
    torch.cuda.synchronize()
    vox_ctx.voxelize(*[f32[k] for k in NAMES], vs, 0.05, flags)
    g32 = vox_ctx.grid()
    vc = int(vox_ctx.stats()["value_count"])
    gd64, gc64 = upstream(vc, 161)
    gd = torch.from_numpy(gd64.astype(np.float32)).cuda()
    gc = torch.from_numpy(gc64.astype(np.float32)).cuda()
    o32 = {k: torch.empty(f32[k].shape, dtype=torch.float32, device="cuda") for k in NAMES}
    vox_ctx.backward(*[f32[k] for k in NAMES], gd, gc, o32)
    vox_ctx.voxelize(*[bf[k] for k in NAMES], vs, 0.05, flags | FLAG_BF16_INPUTS)
    g16 = vox_ctx.grid()
    assert np.array_equal(g16.buf, g32.buf), "BF16 grid differs from the float grid of the same values"
    o16 = {k: torch.empty(f32[k].shape, dtype=torch.float32, device="cuda") for k in NAMES}
    vox_ctx.backward(*[bf[k] for k in NAMES], gd, gc, o16)
    for k in NAMES:
        assert torch.equal(o16[k], o32[k]), k
    # against FP64: the oracle on the same (bfloat16-representable) values
    p32 = {k: f32[k].cpu().numpy() for k in NAMES}
    ref = smooth_forward(oracle_mod, p32, vs)
    v = ref.values()
    dmax = float(np.abs(v["density64"]).max())
    derr = float(np.abs(g16.density.astype(np.float64) - v["density64"]).max())
    assert derr <= REL * dmax, (derr, dmax)
    an = ref.smooth_grad64(p32, True, gd64.astype(np.float32).astype(np.float64), gc64.astype(np.float32).astype(np.float64))
    for k in NAMES:
        scale = float(np.abs(an[k]).max())
        err = float(np.abs(o16[k].cpu().numpy().astype(np.float64).reshape(an[k].shape) - an[k]).max())
        print(f"bf16 adjoint {k}: max |f32 - f64| = {err:.3g} ({err / scale:.2e} of max)")
        assert err <= REL * scale, (k, err, scale)
    ref.close()


def test_bf16_batch_equals_float_batch(vox_ctx):
    import torch

    from nanovdb_editor.vox import FLAG_BF16_INPUTS, FLAG_RAW_INPUTS

    clouds, start, vs = W.batch_clouds(6, 62, min_n=500, max_n=30_000, vs_min=0.002, vs_max=0.01)
    raw = W.concat(clouds).raw_arrays()
    params = {"means": raw[0], "quats": raw[2], "scales": raw[3], "opacities": raw[1], "colors": raw[4]}
    bf, f32 = _pair(params)
    torch.cuda.synchronize()
    _, goff, _ = vox_ctx.voxelize_batch(*[f32[k] for k in NAMES], start, vs, 0.05, FLAG_RAW_INPUTS)
    a = vox_ctx.grids(goff)
    _, goff16, _ = vox_ctx.voxelize_batch(*[bf[k] for k in NAMES], start, vs, 0.05, FLAG_RAW_INPUTS | FLAG_BF16_INPUTS)
    b = vox_ctx.grids(goff16)
    assert np.array_equal(goff, goff16)
    for x, y in zip(a, b):
        assert np.array_equal(x.buf, y.buf)


def test_adam_bf16_step(vox_ctx):
    import torch

    n = 1_000_003
    rng = np.random.default_rng(63)
    master = rng.standard_normal(n).astype(np.float32)
    m = (0.1 * rng.standard_normal(n)).astype(np.float32)
    v = np.abs(0.01 * rng.standard_normal(n)).astype(np.float32)
    grads = [rng.standard_normal(n).astype(np.float32) for _ in range(3)]
    dm, dmm, dv = (torch.from_numpy(a.copy()).cuda() for a in (master, m, v))
    out = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    lr, b1, b2, eps = 1e-2, 0.9, 0.999, 1e-8
    M, Mm, Mv = master.astype(np.float64), m.astype(np.float64), v.astype(np.float64)
    for t, g in enumerate(grads, start=4):
        torch.cuda.synchronize()
        vox_ctx.adam_bf16(dm, dmm, dv, torch.from_numpy(g).cuda(), out, t, lr, b1, b2, eps)
        torch.cuda.synchronize()
        g64 = g.astype(np.float64)
        Mm = b1 * Mm + (1 - b1) * g64
        Mv = b2 * Mv + (1 - b2) * g64 * g64
        M = M - lr * (Mm / (1 - b1**t)) / (np.sqrt(Mv / (1 - b2**t)) + eps)
    got = dm.cpu().numpy().astype(np.float64)
    assert float(np.abs(got - M).max()) <= 1e-5 * float(np.abs(M).max())
    assert torch.equal(out, dm.to(torch.bfloat16))  # the bfloat16 attributes: the master rounded to nearest even
    from nanovdb_editor.exceptions import PipelineError

    with pytest.raises(PipelineError):
        vox_ctx.adam_bf16(dm, dmm, dv, torch.zeros(3, device="cuda"), out, 1, lr)
