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
