"""The file readers behind raster_file and the fileformat table
(fileformat/FileFormat.cpp:87-205, :754-800), on CPU: valid .npz (stored,
deflated, ZIP64, the "sh" alias) and .ply (both byte orders) files load
exactly; malformed files whose header counts would overflow or overrun the
file are rejected with FALSE instead of being read (no GPU needed: the readers
run before any device work)."""

import ctypes
import os
import struct
import zipfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "nanovdb-editor_b200", "nanovdb_editor", "lib", "libpnanovdbcompute.so")

NAMES = ["means", "opacities", "quaternions", "scales", "sh_0"]


class ComputeArray(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("element_size", ctypes.c_uint64),
        ("element_count", ctypes.c_uint64),
        ("filepath", ctypes.c_char_p),
    ]


LOAD = ctypes.CFUNCTYPE(
    ctypes.c_int32, ctypes.c_char_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.POINTER(ComputeArray))
)


class FileFormat(ctypes.Structure):
    _fields_ = [
        ("interface_pnanovdb_reflect_data_type", ctypes.c_void_p),
        ("can_load_file", ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_char_p)),
        ("load_file", LOAD),
        ("module", ctypes.c_void_p),
    ]


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import build_ext

        build_ext.build()
    return ctypes.CDLL(LIB)


@pytest.fixture(scope="module")
def ff(lib):
    lib.pnanovdb_get_fileformat.restype = ctypes.POINTER(FileFormat)
    return lib.pnanovdb_get_fileformat().contents


@pytest.fixture(scope="module")
def destroy(lib):
    from nanovdb_editor.compute import pnanovdb_Compute

    lib.pnanovdb_get_compute.restype = ctypes.POINTER(pnanovdb_Compute)
    c = lib.pnanovdb_get_compute().contents
    fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(ComputeArray))(ctypes.cast(c.destroy_array, ctypes.c_void_p).value)
    return fn


def load(ff, destroy, path, names=NAMES):
    n = len(names)
    cnames = (ctypes.c_char_p * n)(*[x.encode() for x in names])
    out = (ctypes.POINTER(ComputeArray) * n)()
    ok = ff.load_file(str(path).encode(), n, cnames, out)
    if not ok:
        assert all(not out[i] for i in range(n))
        return None
    res = []
    for i in range(n):
        a = out[i].contents
        assert a.element_size == 4
        buf = (ctypes.c_float * a.element_count).from_address(a.data) if a.element_count else []
        res.append(np.array(buf, dtype=np.float32))
        destroy(out[i])
    return res


def cloud(n=37, seed=3):
    rng = np.random.default_rng(seed)
    return {
        "means": rng.normal(size=(n, 3)).astype(np.float32),
        "opacities": rng.normal(size=(n,)).astype(np.float32),
        "quaternions": rng.normal(size=(n, 4)).astype(np.float32),
        "scales": rng.normal(size=(n, 3)).astype(np.float32),
        "sh_0": rng.normal(size=(n, 3)).astype(np.float32),
        "sh_n": rng.normal(size=(n, 15, 3)).astype(np.float32),
    }


def check_same(got, c, names=NAMES):
    assert got is not None
    for g, nm in zip(got, names):
        np.testing.assert_array_equal(g, c[nm].reshape(-1))


@pytest.mark.parametrize("compressed", [False, True])
def test_npz_stored_and_deflated(tmp_path, ff, destroy, compressed):
    c = cloud()
    p = tmp_path / "g.npz"
    (np.savez_compressed if compressed else np.savez)(p, **c)
    check_same(load(ff, destroy, p, NAMES + ["sh_n"]), c, NAMES + ["sh_n"])
    assert ff.can_load_file(str(p).encode()) == 1
    assert ff.can_load_file(b"x.e57") == 0


def test_npz_zip64_and_sh_alias(tmp_path, ff, destroy):
    c = cloud(11)
    sh = np.concatenate([c["sh_0"][:, None, :], c["sh_n"]], axis=1)  # (G, 16, 3)
    p = tmp_path / "z.npz"
    with zipfile.ZipFile(p, "w", compression=zipfile.ZIP_DEFLATED) as z:
        for nm in ["means", "opacities", "quaternions", "scales"]:
            with z.open(nm + ".npy", "w", force_zip64=True) as f:
                np.lib.format.write_array(f, c[nm])
        with z.open("sh.npy", "w", force_zip64=True) as f:
            np.lib.format.write_array(f, sh)
    check_same(load(ff, destroy, p, NAMES + ["sh_n"]), c, NAMES + ["sh_n"])


def test_npz_missing_array(tmp_path, ff, destroy):
    c = cloud()
    del c["scales"]
    p = tmp_path / "m.npz"
    np.savez(p, **c)
    assert load(ff, destroy, p) is None


def write_ply(path, c, big=False, count=None, props_extra=()):
    n = c["means"].shape[0]
    props = ["x", "y", "z", "opacity", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2", "f_dc_0", "f_dc_1", "f_dc_2"]
    props += list(props_extra)
    rows = np.concatenate([c["means"], c["opacities"][:, None], c["quaternions"], c["scales"], c["sh_0"]], axis=1)
    rows = np.concatenate([rows, np.zeros((n, len(props_extra)), np.float32)], axis=1)
    hdr = "ply\nformat binary_%s_endian 1.0\nelement vertex %d\n" % ("big" if big else "little", n if count is None else count)
    hdr += "".join("property float %s\n" % p for p in props) + "end_header\n"
    with open(path, "wb") as f:
        f.write(hdr.encode())
        f.write(rows.astype(">f4" if big else "<f4").tobytes())


@pytest.mark.parametrize("big", [False, True])
def test_ply_both_byte_orders(tmp_path, ff, destroy, big):
    c = cloud(23)
    p = tmp_path / "g.ply"
    write_ply(p, c, big=big)
    check_same(load(ff, destroy, p), c)


@pytest.mark.parametrize("count", [2**62 + 1, 2**40, 2**64 - 1, 24])
def test_ply_vertex_count_beyond_file(tmp_path, ff, destroy, count):
    # 2^62 + 1 vertices of 4 properties wrap nprop * count in 64 bits; 2^40 would
    # need 56 TB; 24 is one row more than the file holds
    c = cloud(23)
    p = tmp_path / "bad.ply"
    write_ply(p, c, count=count)
    assert load(ff, destroy, p) is None


def test_ply_bad_count_text(tmp_path, ff, destroy):
    p = tmp_path / "neg.ply"
    p.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex -5\nproperty float x\nend_header\n" + b"\0" * 64)
    assert load(ff, destroy, p, ["means"]) is None


def npy_bytes(shape_text, payload=b""):
    hdr = "{'descr': '<f4', 'fortran_order': False, 'shape': %s, }" % shape_text
    hdr = hdr + " " * ((64 - (10 + len(hdr) + 1) % 64) % 64) + "\n"
    return b"\x93NUMPY\x01\x00" + struct.pack("<H", len(hdr)) + hdr.encode() + payload


@pytest.mark.parametrize(
    "shape",
    [
        "(4611686018427387905, 4)",  # count * 4 bytes wraps
        "(4294967296, 4294967297)",  # the shape product itself wraps
        "(99999999999999999999999,)",  # a dimension above 2^64
        "(1000000000,)",  # more floats than the entry holds
    ],
)
def test_npy_shape_beyond_entry(tmp_path, ff, destroy, shape):
    p = tmp_path / "s.npz"
    with zipfile.ZipFile(p, "w") as z:
        z.writestr("means.npy", npy_bytes(shape, b"\0" * 64))
    assert load(ff, destroy, p, ["means"]) is None


def test_zip_entry_sizes_beyond_file(tmp_path, ff, destroy):
    c = cloud(5)
    good = tmp_path / "g.npz"
    np.savez(good, means=c["means"])
    data = bytearray(good.read_bytes())
    # central directory entry: compressed / uncompressed sizes -> 0xFFFFFFF0
    cd = data.rfind(b"PK\x01\x02")
    data[cd + 20 : cd + 28] = struct.pack("<II", 0xFFFFFFF0, 0xFFFFFFF0)
    bad = tmp_path / "b.npz"
    bad.write_bytes(bytes(data))
    assert load(ff, destroy, bad, ["means"]) is None
    # local header offset beyond the file
    data = bytearray(good.read_bytes())
    data[cd + 42 : cd + 46] = struct.pack("<I", 0x7FFFFFFF)
    bad.write_bytes(bytes(data))
    assert load(ff, destroy, bad, ["means"]) is None


def test_zip64_extra_field_past_its_length(tmp_path, ff, destroy):
    c = cloud(5)
    good = tmp_path / "g.npz"
    np.savez(good, means=c["means"])
    data = bytearray(good.read_bytes())
    cd = data.rfind(b"PK\x01\x02")
    # sizes marked as ZIP64 but an extra block that claims more bytes than the field has
    nlen = struct.unpack("<H", data[cd + 28 : cd + 30])[0]
    data[cd + 20 : cd + 28] = struct.pack("<II", 0xFFFFFFFF, 0xFFFFFFFF)
    extra = struct.pack("<HH", 1, 200) + b"\xff" * 4
    data[cd + 30 : cd + 32] = struct.pack("<H", len(extra))
    data[cd + 46 + nlen : cd + 46 + nlen] = extra
    eocd = data.rfind(b"PK\x05\x06")
    cd_size = struct.unpack("<I", data[eocd + 12 : eocd + 16])[0]
    data[eocd + 12 : eocd + 16] = struct.pack("<I", cd_size + len(extra))
    bad = tmp_path / "x.npz"
    bad.write_bytes(bytes(data))
    assert load(ff, destroy, bad, ["means"]) is None


def test_corrupt_deflate_and_crc(tmp_path, ff, destroy):
    c = cloud(50)
    good = tmp_path / "g.npz"
    np.savez_compressed(good, means=c["means"])
    raw = good.read_bytes()
    lh = raw.find(b"PK\x03\x04")
    start = lh + 30 + struct.unpack("<H", raw[lh + 26 : lh + 28])[0] + struct.unpack("<H", raw[lh + 28 : lh + 30])[0]
    data = bytearray(raw)
    data[start + 20] ^= 0x5A  # corrupt the deflate stream
    bad = tmp_path / "d.npz"
    bad.write_bytes(bytes(data))
    assert load(ff, destroy, bad, ["means"]) is None
    np.savez(good, means=c["means"])
    data = bytearray(good.read_bytes())
    lh = data.find(b"PK\x03\x04")
    start = lh + 30 + struct.unpack("<H", data[lh + 26 : lh + 28])[0] + struct.unpack("<H", data[lh + 28 : lh + 30])[0]
    data[start + 200] ^= 1  # a stored float bit: the CRC no longer matches
    bad.write_bytes(bytes(data))
    assert load(ff, destroy, bad, ["means"]) is None


def test_truncated_files(tmp_path, ff, destroy):
    c = cloud(9)
    good = tmp_path / "g.npz"
    np.savez(good, **c)
    raw = good.read_bytes()
    for cut in (0, 10, len(raw) // 2, len(raw) - 1):
        p = tmp_path / ("t%d.npz" % cut)
        p.write_bytes(raw[:cut])
        assert load(ff, destroy, p) is None
    assert load(ff, destroy, tmp_path / "absent.npz") is None


def test_raster_file_rejects_malformed_file(tmp_path, lib):
    """raster_file through the reference's table: a file whose vertex count
    wraps the row size returns FALSE (and logs) instead of overrunning."""
    from nanovdb_editor.compute import pnanovdb_ComputeArray
    from nanovdb_editor.raster import pnanovdb_Raster

    lib.pnanovdb_get_raster.restype = ctypes.POINTER(pnanovdb_Raster)
    r = lib.pnanovdb_get_raster().contents
    p = tmp_path / "bad.ply"
    write_ply(p, cloud(4), count=2**62 + 1)
    out = ctypes.POINTER(pnanovdb_ComputeArray)()
    ok = r.raster_file(ctypes.addressof(r), r.compute, None, str(p).encode(), 0.01, ctypes.byref(out), None, None, None, None, None, None)
    assert ok == 0 and not out
