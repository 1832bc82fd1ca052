"""The online launch tuner (OnlineChoice): per size class the first call is a
warm-up, the next calls try each leaf-walk variant (4 and 3 CTAs per SM) once,
and later calls run the faster one.  Every variant gives the same grid."""

import numpy as np
import pytest

from nanovdb_editor import workloads as W

pytestmark = pytest.mark.gpu


def test_walk_variants_tried_after_warmup_and_identical():
    from nanovdb_editor.vox import VoxContext

    cloud = W.cluster_cloud(60_000, 71, clusters=8)
    ctx = VoxContext(0)
    try:
        grids, per_sm = [], []
        for _ in range(5):
            g = ctx.voxelize_host(cloud["means"], cloud["quats"], cloud["scales"], cloud["opacities"], cloud["colors"], 0.002)
            grids.append(g.buf.copy())
            per_sm.append(int(ctx.stats()["walk_ctas_per_sm"]))
        # warm-up (variant 0), then variant 0 and variant 1 once each, then the faster of the two
        assert per_sm[0] == per_sm[1] and per_sm[2] != per_sm[1], per_sm
        assert per_sm[3] == per_sm[4] and per_sm[3] in (per_sm[1], per_sm[2]), per_sm
        for b in grids[1:]:
            assert np.array_equal(b, grids[0])
    finally:
        ctx.close()
