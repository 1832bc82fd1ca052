"""The float density / colour channels of the oracle against its FP64 restatement.

The float channels' local AABB is leaf-relative (the leaf corner's offset
fma(o, vs, -mu) rounded once, then scaled voxel steps), so its rounding error is
relative to the Gaussian's neighbourhood, not to the coordinates' magnitude: the
density stays within 1e-5 of the grid's maximum of the FP64 evaluation (the 64
lattice samples in double) also far from the origin.  The CUDA path evaluates
the same float operations (tests/test_gpu_parity.py compares it with the oracle
bit for bit), so this bounds its error too.
"""

import numpy as np
import pytest

from nanovdb_editor import workloads as W

TOL_REL_MAX = 1e-5


def _far(n, seed, shift):
    c = W.plain_cloud(n, seed)
    c["means"] += np.float32(shift)
    return c


@pytest.mark.parametrize(
    "make,vs",
    [
        (lambda: W.plain_cloud(3000, 31), 0.01),
        (lambda: W.cluster_cloud(4000, 32, clusters=4), 0.002),
        (lambda: _far(2000, 33, 640.0), 0.01),
        (lambda: _far(2000, 34, -600.0), 0.01),
    ],
)
def test_float_channels_within_tolerance_of_fp64(oracle_mod, make, vs):
    cloud = make()
    ref = oracle_mod.OracleResult(cloud, vs, 0.05, window_mode=0)
    assert ref.counts["error"] == 0 and ref.counts["V"] > 0
    v = ref.values()
    dmax = float(np.abs(v["density64"]).max())
    err = float(np.abs(v["density"].astype(np.float64) - v["density64"]).max())
    assert err <= TOL_REL_MAX * dmax, (err, dmax)
    w = v["density64"] > 1e-3 * dmax
    err_c = float(np.abs(v["color"].astype(np.float64)[w] - v["color64"][w]).max())
    assert err_c <= 1e-4, err_c
    ref.close()


def _ulp(y):
    y = np.abs(y).astype(np.float32)
    return np.maximum(np.spacing(y).astype(np.float64), 2.0 ** -149)


def test_channel_math_accuracy(oracle_mod):
    # vox_expf_ch / vox_logf_ch / vox_powf_ch against double precision over their
    # domain (x <= 0, b in (0, 1], e > 0): exp within 1.5 ulp, log within 1.5 ulp
    # of max(|log b|, 1/2), b^e within 1.2e-7 absolute (what the alpha 1 - b^e sees)
    rng = np.random.default_rng(77)
    n = 2_000_000
    u = rng.random(n)
    x = (-87.0 * u * u).astype(np.float32)
    b = np.where(u < 0.5, np.ldexp(1.0 + u, -(48 * u).astype(np.int64)), u).clip(2.0 ** -24, 1.0).astype(np.float32)
    e = (0.05 + 20.0 * rng.random(n) ** 2).astype(np.float32)
    ex, lg, pw = oracle_mod.chan_math(x, b, e)
    ref_e = np.exp(x.astype(np.float64))
    assert float(np.max(np.abs(ex - ref_e) / _ulp(ref_e))) <= 1.5
    ref_l = np.log(b.astype(np.float64))
    assert float(np.max(np.abs(lg - ref_l) / _ulp(np.maximum(np.abs(ref_l), 0.5)))) <= 1.5
    ref_p = np.power(b.astype(np.float64), e.astype(np.float64))
    assert float(np.max(np.abs(pw - ref_p))) <= 1.2e-7
    assert oracle_mod.chan_math(np.zeros(1), np.zeros(1), np.ones(1))[2][0] == 0.0  # 0^e
    assert oracle_mod.chan_math(np.zeros(1), np.ones(1), np.ones(1) * 3)[2][0] == 1.0  # 1^e
