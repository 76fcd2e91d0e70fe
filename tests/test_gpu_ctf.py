"""ctfphaseflip on the GPU through the C ABI against the oracle's restatement of
apps/ctfphaseflip/src/main.rs (itself pinned to an independent numpy FP64 form
in test_ctf_oracle.py).

Tolerance: rel-L2 <= 1e-5 of the corrected stack (the FFTs round differently;
the CTF sign decisions, taken in f64 by both, agree), header statistics within
1e-5.  The per-strip seam (GpuCtfSession::correct_strip, ctf_correct.wgsl in
f32) must give the oracle's f32 restatement except at frequencies whose CTF is
within the f32 rounding of sin/cos of zero: at most 1 in 10^4 flips differ.
"""
import numpy as np
import pytest

import oracle as O
import tiltgpu as T
from tgutil import rel_l2

pytestmark = pytest.mark.gpu


def stack(nz, ny, nx, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((nz, ny, nx)).astype(np.float64)
    k = np.fft.rfftfreq(nx)
    y = np.fft.irfft(np.fft.rfft(x, axis=-1) / (1.0 + (k / 0.1) ** 2), n=nx, axis=-1)
    return (y / y.std() + 5.0).astype(np.float32)


CASES = [
    (dict(pixel_size=2.0, strip_width=32), (3, 40, 96)),                     # radix rows and columns
    (dict(pixel_size=1.5, strip_width=24, tilt_axis_angle=12.0, amplitude_contrast=0.1), (2, 30, 50)),
    (dict(pixel_size=3.0, strip_width=40, plate_phase=90.0, cuton_freq=0.01, max_strip_width=30), (2, 36, 70)),
    (dict(pixel_size=2.0, strip_width=37), (2, 41, 111)),                    # prime strip sizes: direct DFT
    (dict(pixel_size=1.0, strip_width=256, defocus=-2500.0), (3, 256, 512)),  # automatic maximum width
]


@pytest.mark.parametrize("kw,shape", CASES)
def test_ctf_phaseflip_vs_oracle(kw, shape):
    st_in = stack(*shape, seed=shape[2])
    ang = np.linspace(-45, 45, shape[0]).astype(np.float32)
    out, stats = T.ctf_phaseflip(st_in, ang, **kw)
    okw = dict(kw)
    okw["pixel_a"] = okw.pop("pixel_size")
    p = O.CtfParams(**okw)
    assert T.ctf_strip_width(shape[2], **kw) == O.ctf_strip_width(p, shape[2])
    want, wst = O.ctfphaseflip(p, st_in, ang)
    assert rel_l2(out, want) <= 1e-5, rel_l2(out, want)
    for k in ("amin", "amax", "amean"):
        assert stats[k] == pytest.approx(wst[k], rel=1e-5, abs=1e-6)
    assert not np.array_equal(out, st_in)


def test_ctf_phaseflip_per_view_astigmatism_and_short_tilt_file():
    st_in = stack(4, 32, 64, seed=7)
    ang = np.array([-30.0, 0.0, 30.0], np.float32)  # one view without an angle: tilt 0
    vd = np.array([[-2000, -2600, 30.0], [-2500, -2500, 0.0], [-3000, -2200, -45.0], [-2800, -2800, 0.0]],
                  np.float32)
    out, _ = T.ctf_phaseflip(st_in, ang, view_defocus=vd, pixel_size=2.0, strip_width=32)
    want, _ = O.ctfphaseflip(O.CtfParams(pixel_a=2.0, strip_width=32), st_in, ang, vd)
    assert rel_l2(out, want) <= 1e-5


def test_ctf_strip_seam_vs_shader_restatement():
    rng = np.random.default_rng(8)
    sw, sh = 256, 512
    re, im = rng.standard_normal((2, sh * sw)).astype(np.float32)
    for astig, ta in ((0, 0.0), (1, 0.3)):
        prm = dict(sw=sw, sh=sh, pixel_a=1.7, wavelength=0.019687, cs_a=2.7e7, amp_contrast=0.07,
                   cuton_freq=0.002, defocus1=-28000.0, defocus2=-31000.0, astig_angle_rad=0.5,
                   has_astigmatism=astig, plate_phase_rad=0.0, tilt_axis_rad=ta)
        gr, gi = T.ctf_correct_strip(re, im, **prm)
        wr, wi = O.ctf_correct_strip(re, im, O.CtfStrip(**prm))
        # every value is the input or its negation, the real and imaginary parts together
        assert np.all((gr == re) | (gr == -re)) and np.all((np.sign(gr) == np.sign(re)) == (np.sign(gi) == np.sign(im)))
        differ = np.count_nonzero(gr != wr)
        assert differ <= 1e-4 * gr.size, differ
        assert 0.2 < np.mean(gr != re) < 0.8


def interpolate(entries, n):
    """interpolate_defocus of main.rs:162-209 (f32 lerp between listed views)."""
    out = [None] * n
    for v, d in entries:
        if v < n:
            out[v] = [np.float32(x) for x in d]
    has = [o is not None for o in out]
    res = [list(o) if o is not None else [np.float32(0)] * 3 for o in out]
    for v in range(n):
        if has[v]:
            continue
        b = next((i for i in range(v - 1, -1, -1) if has[i]), None)
        a = next((i for i in range(v + 1, n) if has[i]), None)
        if b is not None and a is not None:
            t = np.float32(v - b) / np.float32(a - b)
            res[v] = [res[b][k] + t * (res[a][k] - res[b][k]) for k in range(3)]
        elif b is not None:
            res[v] = list(res[b])
        elif a is not None:
            res[v] = list(res[a])
    return np.array(res, np.float32)


def test_ctfphaseflip_cli_with_defocus_file(tmp_path):
    import subprocess
    nz, ny, nx = 5, 48, 80
    st_in = stack(nz, ny, nx, seed=9)
    src, tlt, out, df = tmp_path / "in.mrc", tmp_path / "in.tlt", tmp_path / "out.mrc", tmp_path / "def.txt"
    h = bytearray(T.mrc_header_new(nx, ny, nz, "Float"))
    # xlen / mx = 2.5 A per pixel (the header's pixel size)
    np.frombuffer(h, "<f4", 3, 40)[:] = (2.5 * nx, 2.5 * ny, 2.5 * nz)
    T.mrc_write_f32(src, bytes(h), st_in)
    ang = np.array([-40.0, -20.0, 0.0, 20.0, 40.0], np.float32)
    T.write_tilt_file(tlt, ang)
    df.write_text("# view def1 def2 astig\n0 -2000 -2400 30\n\n3 -3000\n")
    r = subprocess.run([T.CTF_CLI_PATH, "-i", src, "-o", out, "-t", tlt, "--defocus-file", df, "-w", "32"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    info, got = T.mrc_read(out)
    assert (info.nx, info.ny, info.nz, info.mode) == (nx, ny, nz, 2)
    assert b"ctfphaseflip: CTF phase correction (2D strips)" in bytes(info.header[224:304])
    vd = interpolate([(0, (-2000, -2400, 30)), (3, (-3000, -3000, 0))], nz)
    want, wst = O.ctfphaseflip(O.CtfParams(pixel_a=2.5, strip_width=32), st_in, T.read_tilt_file(tlt), vd)
    assert rel_l2(got.reshape(want.shape), want) <= 1e-5
    assert info.amean == pytest.approx(wst["amean"], rel=1e-5)
