"""The reference-facing entry points (the pnanovdb_raster_t table) against the
oracle: raster_to_nanovdb_from_arrays (raw arrays, raster/RasterUtils.cpp:400-415),
raster_to_nanovdb (activated arrays, raster/Raster.cpp:560-672) and raster_file
(an .npz of raw arrays, raster/RasterUtils.cpp:295-395).  They return what the
reference's entries return - the node2 tree in the reference's node order (its
window-by-window build) and the RGBA8 values, without the float channels - so
the node2 region, bbox and RGBA8 values must equal the oracle's window-mode
restatement byte for byte; the caller's arrays must come back unchanged."""

import numpy as np
import pytest

from nanovdb_editor import workloads as W
from nanovdb_editor.grid import NodeGrid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def raster(vox_ctx):
    from nanovdb_editor import Compute, Raster

    compute = Compute(device_index=0)
    return compute, Raster(compute)


def _grid(compute, arr) -> NodeGrid:
    with compute.mapped_array(arr, np.uint8) as view:
        buf = view.copy()
    compute.destroy_array(arr)
    return NodeGrid(buf)


def _against_oracle(g: NodeGrid, activated, vs, oracle_mod):
    ref = oracle_mod.OracleResult(activated, vs, 0.05, window_mode=1)
    assert ref.counts["error"] == 0 and ref.counts["V"] > 0
    assert int(g.header["node_order"]) == 1
    assert np.array_equal(g.node2, ref.node2())
    v = ref.values()
    np.testing.assert_array_equal(g.rgba8, v["rgba8"])
    assert g.density is None and g.color is None  # RGBA8 only, as the reference returns
    assert int(g.header["grid_bytes"]) == int(g.header["rgba8_offset"]) + 4 * g.value_count
    assert g.buf.size >= int(g.header["grid_bytes"])
    np.testing.assert_array_equal(g.bbox, ref.bbox())
    ref.close()


def test_raster_to_nanovdb_from_arrays(raster, oracle_mod):
    compute, r = raster
    raw = W.plain_cloud(60_000, 41).raw_arrays()  # [means, logits, quats, log scales, sh0, sh_n]
    before = [a.copy() for a in raw]
    arrays = [compute.create_array(a) for a in raw]
    g = _grid(compute, r.raster_to_nanovdb_from_arrays(0.01, arrays))
    for a in arrays:
        compute.destroy_array(a)
    for a, b in zip(raw, before):
        np.testing.assert_array_equal(a, b)  # the reference modifies its inputs in place; this build does not
    _against_oracle(g, oracle_mod.preprocess(raw), 0.01, oracle_mod)


def test_raster_to_nanovdb_activated(raster, oracle_mod):
    compute, r = raster
    cloud = W.cluster_cloud(30_000, 42, clusters=4)
    empty = np.zeros(0, np.float32)
    arrs = {k: compute.create_array(np.ascontiguousarray(cloud[k])) for k in ("means", "quats", "scales", "colors", "opacities")}
    sh0, shn = compute.create_array(empty), compute.create_array(empty)
    out = r.raster_to_nanovdb(0.004, arrs["means"], arrs["quats"], arrs["scales"], arrs["colors"], sh0, shn, arrs["opacities"])
    g = _grid(compute, out)
    _against_oracle(g, cloud, 0.004, oracle_mod)


def test_raster_file(raster, oracle_mod, tmp_path):
    compute, r = raster
    raw = W.plain_cloud(20_000, 43).raw_arrays()
    path = tmp_path / "splats.npz"
    np.savez(path, means=raw[0], opacities=raw[1], quaternions=raw[2], scales=raw[3], sh_0=raw[4], sh_n=raw[5])
    g = _grid(compute, r.raster_file(str(path), 0.01))
    _against_oracle(g, oracle_mod.preprocess(raw), 0.01, oracle_mod)


def test_raster_file_missing_array(raster, tmp_path):
    compute, r = raster
    raw = W.plain_cloud(100, 44).raw_arrays()
    path = tmp_path / "bad.npz"
    np.savez(path, means=raw[0], opacities=raw[1])
    with pytest.raises(RuntimeError):
        r.raster_file(str(path), 0.01)
