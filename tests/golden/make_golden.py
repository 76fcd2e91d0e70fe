"""Extract the boundary test vectors of the reference's own unit tests.

Reads crates/imod-mrc/src/tests.rs, crates/imod-transforms/src/tests.rs and
crates/imod-math/src/tests.rs of the imod-rs source tree (its root is given as argv[1], or in the environment
variable IMOD_RS_SRC) and
writes tests/golden/reference_vectors.json: for each reference test the
constructor arguments, labels, statistics and the data-generating expression,
with the file:line it came from.  Every expected pattern is asserted, so a
change in the reference makes this script fail instead of producing a silently
different fixture.  Run it where the reference is mounted; the JSON is
committed and is all the tests read.
"""
import json
import os
import re
import sys

SRC = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IMOD_RS_SRC", "")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")


def body(text, name):
    m = re.search(r"fn\s+" + name + r"\s*\(\)\s*\{", text)
    assert m, name
    start = m.end()
    depth, i = 1, start
    while depth:
        depth += {"{": 1, "}": -1}.get(text[i], 0)
        i += 1
    line = text.count("\n", 0, m.start()) + 1
    return text[start:i - 1], line


def one(pattern, s, conv=str):
    m = re.search(pattern, s)
    assert m, pattern
    return conv(m.group(1))


def main():
    if not SRC or not os.path.isdir(SRC):
        sys.exit("usage: make_golden.py <imod-rs source root>  (or set IMOD_RS_SRC)")
    mrc_path = os.path.join(SRC, "crates/imod-mrc/src/tests.rs")
    tlt_path = os.path.join(SRC, "crates/imod-transforms/src/tests.rs")
    mrc = open(mrc_path).read()
    tlt = open(tlt_path).read()
    rel_m = "crates/imod-mrc/src/tests.rs"
    rel_t = "crates/imod-transforms/src/tests.rs"
    out = {}

    b, ln = body(mrc, "header_size_is_1024_bytes")
    args = re.search(r"MrcHeader::new\((\d+),\s*(\d+),\s*(\d+),\s*MrcMode::(\w+)\)", b).groups()
    assert "MrcHeader::SIZE" in b
    out["header_size_is_1024_bytes"] = {"src": f"{rel_m}:{ln}", "dims": [int(a) for a in args[:3]],
                                        "mode": args[3], "size": 1024}

    b, ln = body(mrc, "roundtrip_header")
    args = re.search(r"MrcHeader::new\((\d+),\s*(\d+),\s*(\d+),\s*MrcMode::(\w+)\)", b).groups()
    out["roundtrip_header"] = {
        "src": f"{rel_m}:{ln}", "dims": [int(a) for a in args[:3]], "mode": args[3],
        "label": one(r'add_label\("([^"]*)"\)', b),
        "amin": one(r"header\.amin\s*=\s*(-?[\d.]+);", b, float),
        "amax": one(r"header\.amax\s*=\s*(-?[\d.]+);", b, float),
        "amean": one(r"header\.amean\s*=\s*(-?[\d.]+);", b, float),
        "amean_tol": one(r"read_back\.amean\s*-\s*[\d.]+\)\.abs\(\)\s*<\s*([\de.-]+)", b, float)}

    b, ln = body(mrc, "roundtrip_byte_file")
    assert "(0..nx * ny).map(|i| (i % 256) as f32)" in b
    assert "(0..nx * ny).map(|i| ((i + 128) % 256) as f32)" in b
    out["roundtrip_byte_file"] = {
        "src": f"{rel_m}:{ln}", "nx": one(r"let nx = (\d+);", b, int), "ny": one(r"let ny = (\d+);", b, int),
        "nz": one(r"let nz = (\d+);", b, int), "slices": ["(i % 256)", "((i + 128) % 256)"],
        "finish": [float(x) for x in re.search(r"finish\(([-\d.]+),\s*([-\d.]+),\s*([-\d.]+)\)", b).groups()]}

    b, ln = body(mrc, "roundtrip_float_file")
    assert "(0..nx * ny).map(|i| i as f32 * 0.1 - 5.0)" in b
    out["roundtrip_float_file"] = {
        "src": f"{rel_m}:{ln}", "nx": one(r"let nx = (\d+);", b, int), "ny": one(r"let ny = (\d+);", b, int),
        "nz": one(r"let nz = (\d+);", b, int), "data": "i * 0.1 - 5.0", "tol": 1e-6,
        "finish": [float(x) for x in re.search(r"finish\(([-\d.]+),\s*([-\d.]+),\s*([-\d.]+)\)", b).groups()]}

    b, ln = body(mrc, "read_big_endian_float_file")
    assert "header.stamp = [0x11, 0x11, 0x00, 0x00];" in b and "(0..npix).map(|i| i as f32 * 1.5)" in b
    out["read_big_endian_float_file"] = {
        "src": f"{rel_m}:{ln}", "nx": one(r"let nx: i32 = (\d+);", b, int),
        "ny": one(r"let ny: i32 = (\d+);", b, int), "nz": one(r"let nz: i32 = (\d+);", b, int),
        "stamp": [0x11, 0x11, 0, 0], "data": "i * 1.5", "tol": 1e-6}

    b, ln = body(mrc, "read_big_endian_short_file")
    assert "(0..npix as i16).map(|i| i * 100 - 1000)" in b
    out["read_big_endian_short_file"] = {
        "src": f"{rel_m}:{ln}", "nx": one(r"let nx: i32 = (\d+);", b, int),
        "ny": one(r"let ny: i32 = (\d+);", b, int), "nz": one(r"let nz: i32 = (\d+);", b, int),
        "data": "i * 100 - 1000"}

    b, ln = body(mrc, "roundtrip_complex_float_file")
    assert "(i as f32 * 0.5, -(i as f32) * 0.3)" in b
    out["roundtrip_complex_float_file"] = {
        "src": f"{rel_m}:{ln}", "nx": one(r"let nx = (\d+);", b, int), "ny": one(r"let ny = (\d+);", b, int),
        "data": "(i * 0.5, -i * 0.3)", "mag_tol": 1e-5}

    b, ln = body(tlt, "tilt_file_roundtrip")
    rng = re.search(r"\((-?\d+)\.\.=(-?\d+)\)\.step_by\((\d+)\)", b).groups()
    out["tilt_file_roundtrip"] = {"src": f"{rel_t}:{ln}", "start": int(rng[0]), "end": int(rng[1]),
                                  "step": int(rng[2]), "tol": one(r"<\s*([\d.]+)\);", b, float)}
    src = open(os.path.join(SRC, "crates/imod-transforms/src/tilt.rs")).read()
    assert '"{:10.2}"' in src
    out["tilt_file_format"] = {"src": "crates/imod-transforms/src/tilt.rs:31", "format": "{:10.2}"}

    # min_max_mean (crates/imod-math/src/stats.rs:844-861): the per-view mean fill and
    # the output header statistics of the tilt path
    mth = open(os.path.join(SRC, "crates/imod-math/src/tests.rs")).read()
    b, ln = body(mth, "test_min_max_mean")
    data = [float(x) for x in one(r"min_max_mean\(&\[([^\]]*)\]\)", b).split(",")]
    out["min_max_mean"] = {
        "src": f"crates/imod-math/src/tests.rs:{ln}", "data": data,
        "min": one(r"assert_eq!\(min,\s*(-?[\d.]+)\)", b, float),
        "max": one(r"assert_eq!\(max,\s*(-?[\d.]+)\)", b, float),
        "mean_num": one(r"mean\s*-\s*([\d.]+)\s*/", b, float),
        "mean_den": one(r"/\s*([\d.]+)\)\.abs\(\)", b, float),
        "tol": one(r"abs\(\)\s*<\s*([\de.-]+)\)", b, float)}

    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
