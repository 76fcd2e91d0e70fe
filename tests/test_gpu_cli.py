"""The drop-in `tilt` command on a GPU: MRC and .tlt in, MRC out, compared with the
oracle's reconstruction of the same stack (apps/tilt/src/main.rs:540-1095)."""
import subprocess

import numpy as np
import pytest

import oracle as O
import tiltgpu as T
from tgutil import rel_l2, smooth_stack

pytestmark = pytest.mark.gpu


def run(*args):
    return subprocess.run([T.CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("extra,okw", [
    ([], {}),
    (["--sirt", "2", "--xtilt-file", "XT", "--log"], dict(sirt=2, log=True)),
    (["--storage", "fp16", "--radial", "0.3,0.05", "-w", "72"], dict(radial=(0.3, 0.05), width=72)),
])
def test_tilt_cli_matches_oracle(tmp_path, extra, okw):
    nz, ny, nx, thick = 13, 6, 64, 30
    proj = (smooth_stack(nz, ny, nx, seed=61) * 100.0).astype(np.float32)
    ang = np.linspace(-54, 54, nz).astype(np.float32)
    src, tlt, out = tmp_path / "in.mrc", tmp_path / "in.tlt", tmp_path / "out.rec"
    T.mrc_write_f32(src, T.mrc_header_new(nx, ny, nz, "Float"), proj)
    T.write_tilt_file(tlt, ang)
    args = ["-i", src, "-o", out, "-t", tlt, "-z", thick]
    xt = None
    if "XT" in extra:
        xt = np.full(nz, 1.5, np.float32)
        xf = tmp_path / "x.txt"
        open(xf, "w").write("\n".join("%.1f" % v for v in xt) + "\n")
        extra = [xf if e == "XT" else e for e in extra]
    r = run(*args, *extra)
    assert r.returncode == 0, r.stderr
    info, vol = T.mrc_read(out)
    onx = okw.get("width", nx)
    assert (info.nx, info.ny, info.nz, info.mode) == (onx, thick, ny, 2)
    kw = dict(okw)
    kw.setdefault("radial", (0.35, 0.05))
    if xt is not None:
        kw["xtilt"] = xt
    ref, rst = O.run(O.Params(nx, ny, nz, ang, thickness=thick, **kw), proj, "64g" if "fp16" in extra else 32)
    tol = 2e-3 if "fp16" in extra else 1e-5
    assert rel_l2(vol.reshape(ref.shape), ref) <= tol
    assert abs(info.amean - rst["amean"]) <= 10 * tol * max(1.0, abs(rst["amean"]))


@pytest.mark.parametrize("chunk_kb", [131072, 4])
def test_tilt_cli_mode_12_and_chunked_io(tmp_path, chunk_kb):
    # --mode 12 (an addition: half output at half the bytes, readable by the reference's
    # read_slice_f32) must equal the float output rounded to nearest even; a 4 KB staging
    # chunk makes both the read and the write pipelines take many chunks
    nz, ny, nx, thick = 17, 9, 64, 30
    proj = (smooth_stack(nz, ny, nx, seed=62) * 100.0).astype(np.float32)
    ang = np.linspace(-54, 54, nz).astype(np.float32)
    src, tlt = tmp_path / "in.mrc", tmp_path / "in.tlt"
    T.mrc_write_f32(src, T.mrc_header_new(nx, ny, nz, "Float"), proj)
    T.write_tilt_file(tlt, ang)
    outs = {}
    for mode in (2, 12):
        out = tmp_path / f"out{mode}.rec"
        r = run("-i", src, "-o", out, "-t", tlt, "-z", thick, "--mode", mode, "--io-chunk-kb", chunk_kb)
        assert r.returncode == 0, r.stderr
        outs[mode] = T.mrc_read(out)
    i2, v2 = outs[2]
    i12, v12 = outs[12]
    assert i12.mode == 12 and (i12.nx, i12.ny, i12.nz) == (i2.nx, i2.ny, i2.nz)
    assert (i12.amin, i12.amax, i12.amean) == (i2.amin, i2.amax, i2.amean)
    np.testing.assert_array_equal(v12, v2.astype(np.float16).astype(np.float32))
    ref, _ = O.run(O.Params(nx, ny, nz, ang, thickness=thick), proj, 32)
    assert rel_l2(v2.reshape(ref.shape), ref) <= 1e-5


def test_tilt_cli_checkpoint_and_resume(tmp_path):
    # --checkpoint writes the SIRT state every K iterations (an addition); --resume from
    # the last one finishes the run: both give the uninterrupted run's file byte for byte
    nz, ny, nx, thick = 15, 8, 64, 30
    proj = (smooth_stack(nz, ny, nx, seed=63) * 100.0 + 500.0).astype(np.float32)
    ang = np.linspace(-56, 56, nz).astype(np.float32)
    src, tlt = tmp_path / "in.mrc", tmp_path / "in.tlt"
    T.mrc_write_f32(src, T.mrc_header_new(nx, ny, nz, "Float"), proj)
    T.write_tilt_file(tlt, ang)
    base = ["-i", src, "-t", tlt, "-z", thick, "--sirt", "5", "--sirt-relax", "0.3", "--log",
            "--storage", "fp16"]
    a, b, c, ck = (tmp_path / n for n in ("a.rec", "b.rec", "c.rec", "state.mrc"))
    r = run(*base, "-o", a)
    assert r.returncode == 0, r.stderr
    r = run(*base, "-o", b, "--checkpoint", ck, "--checkpoint-every", "2")
    assert r.returncode == 0, r.stderr
    assert "after 4 of 5 iterations" in r.stderr
    info, state = T.mrc_read(ck)
    assert (info.nx, info.ny, info.nz, info.mode) == (nx, thick, ny, 2)
    r = run(*base, "-o", c, "--resume", ck)
    assert r.returncode == 0, r.stderr
    assert "resuming SIRT after 4 of 5" in r.stderr
    assert a.read_bytes() == b.read_bytes() == c.read_bytes()
    # a state of another geometry is refused
    r = run(*base[:4], "-z", thick + 2, *base[6:], "-o", tmp_path / "d.rec", "--resume", ck)
    assert r.returncode == 1 and "does not match" in r.stderr
