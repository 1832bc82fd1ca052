"""The FP64 adjoint of the differentiable channels, pinned by FP64 central
finite differences (h = 1e-6) on sampled parameters.

The channels: density = sum over the pair set of K = max(op exp(-|z|^2/2) - 0.01, 0),
z = S^-1 R^T (x - mu) at the voxel centre; colour = sum K rgb.  The oracle's
float channels are the product's bit-for-bit; its FP64 channels and FP64
gradient are the reference the GPU adjoint is compared with.
"""

import numpy as np
import pytest

from nanovdb_editor import workloads as W

H = 1e-6
REL = 1e-5  # |fd - analytic| <= REL * max |analytic| of the parameter family
FAMILIES = {"means": (0, 3), "quats": (3, 7), "scales": (7, 10), "opacities": (10, 11), "colors": (11, 14)}


def raw_params(cloud, seed):
    """The reference's array form (log-scales, logits, SH0) with quaternions of
    non-unit norm, so the normalisation is part of the chain."""
    rng = np.random.default_rng(seed)
    means, logit, quats, log_s, sh0, _ = cloud.raw_arrays()
    quats = (quats * rng.uniform(0.5, 2.0, (quats.shape[0], 1))).astype(np.float32)
    return {"means": means, "quats": quats, "scales": log_s, "opacities": logit, "colors": sh0}


def smooth_forward(oracle_mod, params, vs):
    act = oracle_mod.preprocess([params["means"], params["opacities"], params["quats"], params["scales"], params["colors"]])
    act["colors"] = act["colors"]
    return oracle_mod.OracleResult(act, vs, 0.05, window_mode=oracle_mod.OV_MODE_SMOOTH)


def upstream(vc, seed):
    rng = np.random.default_rng(seed)
    gd = rng.standard_normal(vc)
    gc = rng.standard_normal((vc, 3))
    gd[:2] = 0.0
    gc[:2] = 0.0
    return gd, gc


def theta_of(params, g):
    return np.concatenate([
        params["means"][g].astype(np.float64),
        params["quats"][g].astype(np.float64),
        params["scales"][g].astype(np.float64),
        [float(params["opacities"][g])],
        params["colors"][g].astype(np.float64),
    ])


def flat_grad(grads, g):
    return np.concatenate([grads["means"][g], grads["quats"][g], grads["scales"][g], [grads["opacities"][g]], grads["colors"][g]])


def test_smooth_channels_fp64(oracle_mod):
    cloud = W.cluster_cloud(3000, 21, clusters=3)
    params = raw_params(cloud, 21)
    ref = smooth_forward(oracle_mod, params, 0.004)
    v = ref.values()
    assert ref.counts["V"] > 0
    dmax = float(np.abs(v["density64"]).max())
    assert float(np.abs(v["density"] - v["density64"]).max()) <= 1e-5 * dmax
    cmax = float(np.abs(v["color64"]).max())
    assert float(np.abs(v["color"] - v["color64"]).max()) <= 1e-5 * cmax
    ref.close()


@pytest.mark.parametrize("seed", [31, 32])
def test_oracle_adjoint_matches_central_differences(oracle_mod, seed):
    cloud = W.cluster_cloud(1500, seed, clusters=2)
    params = raw_params(cloud, seed)
    vs = 0.004
    ref = smooth_forward(oracle_mod, params, vs)
    gd, gc = upstream(ref.counts["value_count"], seed + 100)
    an = ref.smooth_grad64(params, True, gd, gc)
    scale = {k: float(np.abs(an[k]).max()) for k in FAMILIES}
    assert all(s > 0 for s in scale.values())
    _, ids = ref.pairs()
    active = np.unique(ids)
    rng = np.random.default_rng(seed + 200)
    checked = kinks = 0
    worst = 0.0
    while checked < 256:
        assert kinks <= 64, "too many samples straddle a kink"
        g = int(rng.choice(active))
        i = int(rng.integers(0, 14))
        fam = next(k for k, (a, b) in FAMILIES.items() if a <= i < b)
        th = theta_of(params, g)

        def fd(h):
            tp, tm = th.copy(), th.copy()
            tp[i] += h
            tm[i] -= h
            return (ref.smooth_loss64(tp, True, gd, gc) - ref.smooth_loss64(tm, True, gd, gc)) / (2 * h)

        f1, f2 = fd(H), fd(H / 2)
        if abs(f1 - f2) > 1e-7 * scale[fam]:
            kinks += 1  # the sample straddles the K = 0 boundary of some voxel
            continue
        a = flat_grad(an, g)[i]
        err = abs(f1 - a) / scale[fam]
        worst = max(worst, err)
        assert err <= REL, (g, i, fam, f1, a, scale[fam])
        checked += 1
    ref.close()
    assert worst <= REL
