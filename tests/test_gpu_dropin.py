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


def _write_ply(path, raw, big_endian=False, extra=()):
    """A binary Gaussian-splat .ply as 3DGS tools write it: per vertex x y z,
    normals, f_dc_0..2, f_rest_0..44, opacity, scale_0..2, rot_0..3 (float32)."""
    means, logits, quats, log_scales, sh0, shn = raw
    n = means.shape[0]
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
    names += [f"f_rest_{i}" for i in range(45)] + ["opacity", "scale_0", "scale_1", "scale_2"]
    names += ["rot_0", "rot_1", "rot_2", "rot_3"] + list(extra)
    rest = shn.reshape(n, 45) if shn.size == 45 * n else np.zeros((n, 45), np.float32)
    cols = [means, np.zeros((n, 3), np.float32), sh0.reshape(n, 3), rest, logits.reshape(n, 1),
            log_scales.reshape(n, 3), quats.reshape(n, 4)] + [np.zeros((n, 1), np.float32)] * len(extra)
    rows = np.concatenate(cols, axis=1).astype(">f4" if big_endian else "<f4")
    fmt = "binary_big_endian" if big_endian else "binary_little_endian"
    head = f"ply\nformat {fmt} 1.0\nelement vertex {n}\n" + "".join(f"property float {c}\n" for c in names)
    head += "end_header\n"
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(rows.tobytes())


@pytest.mark.parametrize("big_endian", [False, True])
def test_raster_file_ply(raster, oracle_mod, tmp_path, big_endian):
    # fileformat/FileFormat.cpp:205-580: the splat .ply layout raster_file also loads
    compute, r = raster
    raw = W.plain_cloud(20_000, 46).raw_arrays()
    path = tmp_path / "splats.ply"
    _write_ply(path, raw, big_endian)
    g = _grid(compute, r.raster_file(str(path), 0.01))
    _against_oracle(g, oracle_mod.preprocess(raw), 0.01, oracle_mod)


def test_raster_file_rejects_unsupported(raster, tmp_path):
    compute, r = raster
    raw = W.plain_cloud(100, 47).raw_arrays()
    ascii_ply = tmp_path / "a.ply"
    ascii_ply.write_text("ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n0\n")
    with pytest.raises(RuntimeError):
        r.raster_file(str(ascii_ply), 0.01)
    other = tmp_path / "a.xyz"
    other.write_bytes(b"0 0 0\n")
    with pytest.raises(RuntimeError):
        r.raster_file(str(other), 0.01)
    no_scales = tmp_path / "b.ply"
    _write_ply(no_scales, raw)
    data = no_scales.read_bytes().replace(b"property float scale_0", b"property float sxale_0")
    no_scales.write_bytes(data)
    with pytest.raises(RuntimeError):
        r.raster_file(str(no_scales), 0.01)


def test_raster_file_missing_array(raster, tmp_path):
    compute, r = raster
    raw = W.plain_cloud(100, 44).raw_arrays()
    path = tmp_path / "bad.npz"
    np.savez(path, means=raw[0], opacities=raw[1])
    with pytest.raises(RuntimeError):
        r.raster_file(str(path), 0.01)


class _Buffer(__import__("ctypes").Structure):
    """pnanovdb_compute_buffer_t: a device pointer and its size"""

    _fields_ = [("device_ptr", __import__("ctypes").c_void_p), ("size_bytes", __import__("ctypes").c_uint64)]


def _raster_3d(compute, r, ctx, data, vs, words):
    """raster_gaussian_3d into a device buffer of `words` 32-bit words; the buffer's bytes on the host"""
    import ctypes

    import torch

    dev = torch.zeros(words, dtype=torch.int32, device="cuda")
    buf = _Buffer(dev.data_ptr(), 4 * words)
    torch.cuda.synchronize()
    t = r._raster.contents
    t.raster_gaussian_3d(compute.get_compute(), compute.queue(), ctx, vs, data, ctypes.byref(buf), words, None)
    torch.cuda.synchronize()
    return dev.cpu().numpy().view(np.uint8)


def test_gaussian_data_and_raster_gaussian_3d(raster, oracle_mod):
    """create_context / create_gaussian_data / upload_gaussian_data /
    raster_gaussian_3d / destroy_gaussian_data / destroy_context through the
    table (raster/RasterContext.cpp:92-229, raster/Raster.cpp:420-558): the
    device buffer receives the reference's output (node2 in the reference's
    node order and RGBA8 values), equal to the oracle; a buffer too small for
    it is left untouched."""
    compute, r = raster
    t = r._raster.contents
    cloud = W.cluster_cloud(20_000, 48, clusters=3)
    vs = 0.004
    arrs = {k: compute.create_array(np.ascontiguousarray(cloud[k])) for k in ("means", "quats", "scales", "colors", "opacities")}
    empty = compute.create_array(np.zeros(0, np.float32))
    ctx = t.create_context(compute.get_compute(), compute.queue())
    assert ctx
    data = t.create_gaussian_data(compute.get_compute(), compute.queue(), ctx, arrs["means"], arrs["quats"], arrs["scales"],
                                  arrs["colors"], empty, empty, arrs["opacities"], None, None)
    assert data
    t.upload_gaussian_data(compute.get_compute(), compute.queue(), ctx, data)
    out = _raster_3d(compute, r, ctx, data, vs, 16 << 20)
    g = NodeGrid(out)
    _against_oracle(g, cloud, vs, oracle_mod)
    need = int(g.header["grid_bytes"])
    small = _raster_3d(compute, r, ctx, data, vs, (need - 4) // 4)
    assert not small.any()  # too small: logged, nothing written
    t.destroy_gaussian_data(compute.get_compute(), compute.queue(), data)
    t.destroy_context(compute.get_compute(), compute.queue(), ctx)
    for a in list(arrs.values()) + [empty]:
        compute.destroy_array(a)


def test_gaussian_data_from_arrays(raster, oracle_mod):
    """create_gaussian_data_from_arrays (raw arrays, raster/RasterUtils.cpp:208-245)
    with a new context, then raster_gaussian_3d: the reference's preprocessing
    runs in the prep kernel and the result equals the oracle's."""
    import ctypes

    from nanovdb_editor.compute import pnanovdb_ComputeArray

    compute, r = raster
    t = r._raster.contents
    raw = W.plain_cloud(15_000, 49).raw_arrays()
    arrays = [compute.create_array(a) for a in raw]
    Arr = ctypes.POINTER(pnanovdb_ComputeArray)
    arr_c = (Arr * 6)(*[ctypes.pointer(a) for a in arrays])
    data, ctx = ctypes.c_void_p(), ctypes.c_void_p()
    ok = t.create_gaussian_data_from_arrays(ctypes.addressof(t), compute.get_compute(), compute.queue(), arr_c, 6,
                                            ctypes.byref(data), None, ctypes.byref(ctx))
    assert ok == 1 and data.value and ctx.value
    g = NodeGrid(_raster_3d(compute, r, ctx.value, data.value, 0.01, 16 << 20))
    _against_oracle(g, oracle_mod.preprocess(raw), 0.01, oracle_mod)
    t.destroy_gaussian_data(compute.get_compute(), compute.queue(), data.value)
    t.destroy_context(compute.get_compute(), compute.queue(), ctx.value)
    for a in arrays:
        compute.destroy_array(a)


def test_queues_run_concurrently(vox_ctx):
    """Worker threads with their own queues (editor/PipelineRuntime.cpp:416-427)
    each get their own context: two threads voxelizing different clouds at once
    return the same grids as one after the other."""
    import threading

    from nanovdb_editor import Compute, Raster

    computes = [Compute(device_index=0) for _ in range(2)]
    rasters = [Raster(c) for c in computes]
    raws = [W.plain_cloud(40_000, 50 + i).raw_arrays() for i in range(2)]

    def run(i, out):
        c = computes[i]
        arrays = [c.create_array(a) for a in raws[i]]
        for _ in range(3):
            g = _grid(c, rasters[i].raster_to_nanovdb_from_arrays(0.01, arrays))
        out[i] = g.buf.copy()
        for a in arrays:
            c.destroy_array(a)

    serial = [None, None]
    for i in range(2):
        run(i, serial)
    both = [None, None]
    th = [threading.Thread(target=run, args=(i, both)) for i in range(2)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for i in range(2):
        assert np.array_equal(both[i], serial[i])
