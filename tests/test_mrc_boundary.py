"""The MRC / .tlt boundary through the C ABI, pinned to the reference's own tests.

tests/golden/reference_vectors.json holds the parameters of the reference's
unit tests (crates/imod-mrc/src/tests.rs, crates/imod-transforms/src/tests.rs),
extracted by tests/golden/make_golden.py.  The header byte layout is checked
against an independent table of crates/imod-mrc/src/header.rs:10-110.
Host-only: no GPU is needed.
"""
import json
import os
import struct

import numpy as np
import pytest

import tiltgpu as T

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))

# (name, struct code, count) in on-disk order, header.rs:10-110
FIELDS = [("nx", "i", 1), ("ny", "i", 1), ("nz", "i", 1), ("mode", "i", 1), ("nxstart", "i", 1),
          ("nystart", "i", 1), ("nzstart", "i", 1), ("mx", "i", 1), ("my", "i", 1), ("mz", "i", 1),
          ("xlen", "f", 1), ("ylen", "f", 1), ("zlen", "f", 1), ("alpha", "f", 1), ("beta", "f", 1),
          ("gamma", "f", 1), ("mapc", "i", 1), ("mapr", "i", 1), ("maps", "i", 1), ("amin", "f", 1),
          ("amax", "f", 1), ("amean", "f", 1), ("ispg", "i", 1), ("next", "i", 1), ("creatid", "h", 1),
          ("blank", "6s", 1), ("ext_type", "4s", 1), ("nversion", "i", 1), ("blank2", "16s", 1),
          ("nint", "h", 1), ("nreal", "h", 1), ("sub", "h", 1), ("zfac", "h", 1), ("min2", "f", 1),
          ("max2", "f", 1), ("min3", "f", 1), ("max3", "f", 1), ("imod_stamp", "i", 1),
          ("imod_flags", "i", 1), ("idtype", "h", 1), ("lens", "h", 1), ("nd1", "h", 1), ("nd2", "h", 1),
          ("vd1", "h", 1), ("vd2", "h", 1), ("tilt_angles", "6f", 6), ("xorg", "f", 1), ("yorg", "f", 1),
          ("zorg", "f", 1), ("cmap", "4s", 1), ("stamp", "4s", 1), ("rms", "f", 1), ("nlabl", "i", 1),
          ("labels", "800s", 1)]
FMT = "".join(code for _, code, _ in FIELDS)
assert struct.calcsize("<" + FMT) == 1024


def parse(hb, endian="<"):
    vals = struct.unpack(endian + FMT, hb)
    out, i = {}, 0
    for name, code, n in FIELDS:
        out[name] = vals[i:i + n] if n > 1 else vals[i]
        i += n
    return out


def pack(d, endian):
    flat = []
    for name, code, n in FIELDS:
        flat.extend(d[name] if n > 1 else [d[name]])
    return struct.pack(endian + FMT, *flat)


def test_header_size_and_new_defaults():
    g = GOLD["header_size_is_1024_bytes"]
    hb = T.mrc_header_new(*g["dims"], g["mode"])
    assert len(hb) == g["size"] == 1024
    h = parse(hb)
    # MrcHeader::new (header.rs:181-241)
    assert (h["nx"], h["ny"], h["nz"], h["mode"]) == (64, 64, 1, 0)
    assert (h["mx"], h["my"], h["mz"]) == (64, 64, 1)
    assert (h["xlen"], h["ylen"], h["zlen"]) == (64.0, 64.0, 1.0)
    assert (h["alpha"], h["beta"], h["gamma"]) == (90.0, 90.0, 90.0)
    assert (h["mapc"], h["mapr"], h["maps"]) == (1, 2, 3)
    assert h["nversion"] == 20140 and h["rms"] == -1.0 and h["nlabl"] == 0
    assert h["cmap"] == b"MAP " and h["stamp"] == b"\x44\x44\x00\x00"
    assert h["imod_stamp"] == struct.unpack("<i", bytes([0x88, 0x44, 0x00, 0x25]))[0]
    assert h["labels"] == b"\0" * 800


def test_roundtrip_header(tmp_path):
    g = GOLD["roundtrip_header"]
    hb = T.mrc_header_new(*g["dims"], g["mode"], label=g["label"])
    p = tmp_path / "h.mrc"
    T.mrc_write_f32(p, hb, None, (g["amin"], g["amax"], g["amean"]))
    info = T.mrc_info(p)
    assert (info.nx, info.ny, info.nz, info.mode) == (128, 256, 10, 2)
    assert info.amin == g["amin"] and info.amax == g["amax"]
    assert abs(info.amean - g["amean"]) < g["amean_tol"]
    assert info.imod == 1 and info.nlabl == 1
    lab = parse(bytes(info.header))["labels"][:80]
    assert lab.decode().rstrip(" ") == g["label"]
    assert lab[len(g["label"]):] == b" " * (80 - len(g["label"]))  # space padded


def test_roundtrip_byte_file(tmp_path):
    g = GOLD["roundtrip_byte_file"]
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    i = np.arange(nx * ny)
    s0, s1 = (i % 256).astype(np.float32), ((i + 128) % 256).astype(np.float32)
    p = tmp_path / "b.mrc"
    T.mrc_write_f32(p, T.mrc_header_new(nx, ny, nz, "Byte"), np.concatenate([s0, s1]), tuple(g["finish"]))
    info, data = T.mrc_read(p)
    assert (info.nx, info.ny, info.nz) == (nx, ny, nz)
    np.testing.assert_array_equal(data[:nx * ny], s0)
    np.testing.assert_array_equal(data[nx * ny:], s1)


def test_roundtrip_float_file(tmp_path):
    g = GOLD["roundtrip_float_file"]
    nx, ny = g["nx"], g["ny"]
    data = (np.arange(nx * ny, dtype=np.float32) * np.float32(0.1) - np.float32(5.0))
    p = tmp_path / "f.mrc"
    T.mrc_write_f32(p, T.mrc_header_new(nx, ny, 1, "Float"), data, tuple(g["finish"]))
    _, back = T.mrc_read(p)
    assert np.max(np.abs(back - data)) < g["tol"]
    raw = open(p, "rb").read()
    assert len(raw) == 1024 + nx * ny * 4
    np.testing.assert_array_equal(np.frombuffer(raw[1024:], "<f4"), data)


def _be_file(path, nx, ny, mode, payload):
    h = parse(T.mrc_header_new(nx, ny, 1, mode))
    h["stamp"] = bytes([0x11, 0x11, 0, 0])
    open(path, "wb").write(pack(h, ">") + payload)


def test_read_big_endian_float_file(tmp_path):
    g = GOLD["read_big_endian_float_file"]
    nx, ny = g["nx"], g["ny"]
    data = np.arange(nx * ny, dtype=np.float32) * np.float32(1.5)
    p = tmp_path / "be.mrc"
    _be_file(p, nx, ny, "Float", data.astype(">f4").tobytes())
    info, back = T.mrc_read(p)
    assert info.swapped == 1 and (info.nx, info.ny) == (nx, ny)
    assert np.max(np.abs(back - data)) < g["tol"]


def test_read_big_endian_short_file(tmp_path):
    g = GOLD["read_big_endian_short_file"]
    nx, ny = g["nx"], g["ny"]
    data = (np.arange(nx * ny, dtype=np.int16) * 100 - 1000).astype(np.int16)
    p = tmp_path / "bes.mrc"
    _be_file(p, nx, ny, "Short", data.astype(">i2").tobytes())
    info, back = T.mrc_read(p)
    assert info.swapped == 1
    np.testing.assert_array_equal(back, data.astype(np.float32))


def test_unreasonable_dims_trigger_swap_detection(tmp_path):
    # no stamp, but little-endian dims are absurd: read as big-endian (read.rs:36-52)
    h = parse(T.mrc_header_new(6, 5, 1, "Float"))
    h["stamp"] = b"\0\0\0\0"
    data = np.linspace(-1, 1, 30).astype(np.float32)
    p = tmp_path / "bed.mrc"
    open(p, "wb").write(pack(h, ">") + data.astype(">f4").tobytes())
    info, back = T.mrc_read(p)
    assert info.swapped == 1 and (info.nx, info.ny) == (6, 5)
    np.testing.assert_array_equal(back, data)


def test_complex_float_magnitude(tmp_path):
    g = GOLD["roundtrip_complex_float_file"]
    nx, ny = g["nx"], g["ny"]
    i = np.arange(nx * ny, dtype=np.float32)
    re, im = i * np.float32(0.5), -i * np.float32(0.3)
    hb = T.mrc_header_new(nx, ny, 1, "ComplexFloat")
    inter = np.stack([re, im], 1).astype("<f4").tobytes()
    p = tmp_path / "c.mrc"
    open(p, "wb").write(hb + inter)
    _, mag = T.mrc_read(p)
    assert np.max(np.abs(mag - np.sqrt(re * re + im * im))) < g["mag_tol"]


def test_half_float_mode_12(tmp_path):
    vals = np.array([0.0, -0.0, 1.0, -2.5, 65504.0, 6.1035156e-05, 5.9604645e-08, np.inf, 3.0e-6],
                    np.float16)
    p = tmp_path / "h12.mrc"
    open(p, "wb").write(T.mrc_header_new(len(vals), 1, 1, "HalfFloat") + vals.astype("<f2").tobytes())
    _, back = T.mrc_read(p)
    np.testing.assert_array_equal(back, vals.astype(np.float32))


def test_four_bit_and_ushort(tmp_path):
    nx, ny = 5, 2
    raw = bytes([0x21, 0x43, 0x05, 0x87, 0xA9, 0x0B])  # rows of (nx+1)//2 = 3 bytes
    p = tmp_path / "m101.mrc"
    open(p, "wb").write(T.mrc_header_new(nx, ny, 1, "FourBit") + raw)
    _, back = T.mrc_read(p)
    np.testing.assert_array_equal(back, [1, 2, 3, 4, 5, 7, 8, 9, 10, 11])
    u = np.array([0, 1, 65535, 40000], np.uint16)
    p2 = tmp_path / "m6.mrc"
    open(p2, "wb").write(T.mrc_header_new(4, 1, 1, "UShort") + u.astype("<u2").tobytes())
    _, back = T.mrc_read(p2)
    np.testing.assert_array_equal(back, u.astype(np.float32))


def test_extended_header_is_skipped(tmp_path):
    h = parse(T.mrc_header_new(3, 2, 1, "Float"))
    h["next"] = 96
    data = np.arange(6, dtype=np.float32)
    p = tmp_path / "ext.mrc"
    open(p, "wb").write(pack(h, "<") + b"\x7f" * 96 + data.astype("<f4").tobytes())
    _, back = T.mrc_read(p)
    np.testing.assert_array_equal(back, data)


def test_tilt_file_roundtrip_and_format(tmp_path):
    g = GOLD["tilt_file_roundtrip"]
    ang = np.arange(g["start"], g["end"] + 1, g["step"]).astype(np.float32)
    p = tmp_path / "a.tlt"
    T.write_tilt_file(p, ang)
    lines = open(p).read().splitlines()
    assert lines[0] == f"{ang[0]:10.2f}" and all(len(x) == 10 for x in lines)
    back = T.read_tilt_file(p)
    assert len(back) == len(ang) and np.max(np.abs(back - ang)) < g["tol"]


def test_tilt_file_skips_blank_and_unparseable(tmp_path):
    p = tmp_path / "b.tlt"
    open(p, "w").write("  -60.0\n\nabc\n 1e1 \n# c\n+5\n0.5x\n")
    np.testing.assert_array_equal(T.read_tilt_file(p), np.array([-60.0, 10.0, 5.0], np.float32))


def test_tilt_output_header():
    # MrcHeader::new(out_nx, out_nz, out_ny) + lengths + label (apps/tilt/src/main.rs:710-717)
    hin = parse(T.mrc_header_new(100, 80, 41, "Float"))
    hin["xlen"], hin["ylen"] = 250.0, 200.0
    out = parse(T.tilt_output_header(pack(hin, "<"), 120, 30))
    assert (out["nx"], out["ny"], out["nz"], out["mode"]) == (120, 30, 80, 2)
    assert (out["mx"], out["my"], out["mz"]) == (120, 30, 80)
    assert out["xlen"] == np.float32(np.float32(250.0) * np.float32(120) / np.float32(100))
    assert out["ylen"] == np.float32(np.float32(250.0) * np.float32(30) / np.float32(100))
    assert out["zlen"] == 200.0 and out["nlabl"] == 1
    assert out["labels"][:80].decode() == "tilt: 41 projections, thickness 30".ljust(80)


def test_write_mode_12_rounds_to_nearest_even(tmp_path):
    # the writer's f32 -> half conversion (an addition: the reference reads mode 12,
    # crates/imod-mrc/src/read.rs:468-499, but does not write it) against numpy's IEEE
    # round-to-nearest-even: normals, ties, subnormals, the largest half, overflow
    rng = np.random.default_rng(12)
    specials = np.array([0.0, -0.0, 1.0, -2.5, 65504.0, 65519.99, 65520.0, -7e4, 1e-8, 2.9802322e-08,
                         5.9604645e-08, 8.940697e-08, 6.1035156e-05, 6.097e-05, 1.0009766, 1.00146484,
                         np.inf, -np.inf, 3.0e-6], np.float32)
    vals = np.concatenate([specials, rng.standard_normal(4000).astype(np.float32) * 10.0 ** rng.integers(-9, 6, 4000)])
    vals = vals.astype(np.float32)
    n = len(vals)
    p = tmp_path / "w12.mrc"
    T.mrc_write_f32(p, T.mrc_header_new(n, 1, 1, "HalfFloat"), vals)
    info, back = T.mrc_read(p)
    assert info.mode == 12 and os.path.getsize(p) == 1024 + 2 * n
    with np.errstate(over="ignore"):
        want = vals.astype(np.float16)
    np.testing.assert_array_equal(np.fromfile(p, "<u2", offset=1024), want.view("<u2"))
    np.testing.assert_array_equal(back, want.astype(np.float32))
