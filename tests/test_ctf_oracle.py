"""The ctfphaseflip restatement in the oracle (apps/ctfphaseflip/src/main.rs),
checked on the CPU against an independent numpy form of the same steps (FP64,
numpy's FFT) and against properties of the phase flip.  No GPU needed."""
import numpy as np
import pytest

import oracle as O

PI32 = float(np.float32(np.pi))


def numpy_ctfphaseflip(stack, angles, p: O.CtfParams, view_def=None):
    """Direct FP64 restatement of main.rs:385-700 with numpy's FFT."""
    nz, ny, nx = stack.shape
    wl = O.ctf_wavelength(p.voltage)
    cs_a = p.cs * 1e7
    amp = float(np.float32(p.amplitude_contrast))
    ta = float(np.float32(p.tilt_axis_angle)) * PI32 / 180.0
    plate = float(np.float32(p.plate_phase)) * PI32 / 180.0
    sw_px = O.ctf_strip_width(p, nx, view_def)
    px, py = np.cos(ta), np.sin(ta)
    cx, cy = nx / 2.0, ny / 2.0
    ys, xs = np.mgrid[0:ny, 0:nx].astype(np.float64)
    d = (xs - cx) * px + (ys - cy) * py
    corners = [(0, 0), (nx, 0), (0, ny), (nx, ny)]
    dd = [(a - cx) * px + (b - cy) * py for a, b in corners]
    mn, mx = min(dd), max(dd)
    n_strips = int(np.ceil((mx - mn) / sw_px))
    out = np.empty_like(stack, dtype=np.float64)
    for z in range(nz):
        data = stack[z].astype(np.float64)
        tilt = float(np.float32(angles[z])) * PI32 / 180.0 if z < len(angles) else 0.0
        if view_def is not None:
            d1, d2, ast = (float(v) for v in view_def[z])
        else:
            d1 = d2 = float(np.float32(p.defocus))
            ast = 0.0
        d1a, d2a, asr = d1 * 10.0, d2 * 10.0, ast * PI32 / 180.0
        astig = abs(d1a - d2a) > 0.01
        wsum = np.zeros((ny, nx))
        wtot = np.zeros((ny, nx))
        for k in range(n_strips):
            c = mn + (k + 0.5) * sw_px
            dxa = c * float(np.float32(p.pixel_a))
            b1, b2 = d1a + dxa * np.sin(tilt), d2a + dxa * np.sin(tilt)
            lo, hi = c - sw_px / 2.0, c + sw_px / 2.0
            m = (d >= lo) & (d < hi)
            if not m.any():
                continue
            yy, xx = np.nonzero(m)
            y0, y1, x0, x1 = yy.min(), yy.max() + 1, xx.min(), xx.max() + 1
            sh, sw = y1 - y0, x1 - x0
            F = np.fft.fft2(data[y0:y1, x0:x1])
            fy = np.arange(sh, dtype=np.float64)
            fy = np.where(fy <= sh // 2, fy, fy - sh)[:, None]
            fx = np.arange(sw, dtype=np.float64)
            fx = np.where(fx <= sw // 2, fx, fx - sw)[None, :]
            if abs(ta) > 1e-6:
                fx, fy = fx * np.cos(ta) + fy * np.sin(ta), -fx * np.sin(ta) + fy * np.cos(ta)
            pa = float(np.float32(p.pixel_a))
            sx = fx / (sw * pa) + 0 * fy
            sy = fy / (sh * pa) + 0 * fx
            s2 = sx * sx + sy * sy
            if astig:
                da = np.arctan2(sy, sx) - asr
                dfc = b1 * np.cos(da) ** 2 + b2 * np.sin(da) ** 2
            else:
                dfc = b1
            chi = np.pi * wl * s2 * (dfc - 0.5 * cs_a * wl * wl * s2) + plate
            ctf = -np.sin(chi) * np.sqrt(1 - amp * amp) + np.cos(chi) * amp
            flip = (ctf < 0) & (np.sqrt(s2) >= float(np.float32(p.cuton_freq)))
            F = np.where(flip, -F, F)
            v = np.fft.ifft2(F).real
            w = np.maximum(1.0 - np.abs((d[y0:y1, x0:x1] - c) / (sw_px / 2.0)), 0.0) * m[y0:y1, x0:x1]
            wsum[y0:y1, x0:x1] += v * w
            wtot[y0:y1, x0:x1] += w
        out[z] = np.where(wtot > 1e-10, wsum / np.where(wtot > 0, wtot, 1), data)
    return out


def stack(nz, ny, nx, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((nz, ny, nx)) + 5.0).astype(np.float32)


@pytest.mark.parametrize("kw,shape", [
    (dict(pixel_a=2.0, strip_width=32), (3, 40, 96)),
    (dict(pixel_a=1.5, strip_width=24, tilt_axis_angle=12.0, amplitude_contrast=0.1), (2, 30, 50)),
    (dict(pixel_a=3.0, strip_width=40, plate_phase=90.0, cuton_freq=0.01, max_strip_width=30), (2, 36, 70)),
])
def test_ctfphaseflip_matches_numpy_fp64(kw, shape):
    p = O.CtfParams(**kw)
    st = stack(*shape, seed=shape[2])
    ang = np.linspace(-40, 40, shape[0]).astype(np.float32)
    out, stats = O.ctfphaseflip(p, st, ang)
    want = numpy_ctfphaseflip(st, ang, p)
    err = np.linalg.norm(out - want) / np.linalg.norm(want)
    assert err <= 2e-6, err
    assert stats["amin"] == out.min() and stats["amax"] == out.max()


def test_ctfphaseflip_astigmatism_per_view():
    p = O.CtfParams(pixel_a=2.0, strip_width=32)
    st = stack(3, 32, 64, seed=4)
    ang = np.array([-30.0, 0.0, 30.0], np.float32)
    vd = np.array([[-2000, -2600, 30.0], [-2500, -2500, 0.0], [-3000, -2200, -45.0]], np.float32)
    out, _ = O.ctfphaseflip(p, st, ang, vd)
    want = numpy_ctfphaseflip(st, ang, p, vd)
    assert np.linalg.norm(out - want) / np.linalg.norm(want) <= 2e-6


def test_strip_width_automatic_maximum():
    # main.rs:297-320: pixel / (wavelength * max|defocus| / nx), at least 16 px
    p = O.CtfParams(pixel_a=1.0, strip_width=4096, defocus=-3000.0)
    wl = O.ctf_wavelength(300.0)
    assert abs(wl - 0.019687) < 1e-5  # 300 kV electrons
    want = int(max(1.0 / (wl * (30000.0 / 2048)), 16.0))
    assert O.ctf_strip_width(p, 2048) == min(4096, want)
    assert O.ctf_strip_width(O.CtfParams(strip_width=100, max_strip_width=64), 2048) == 64


def test_strip_flip_is_an_involution_and_keeps_low_frequencies():
    rng = np.random.default_rng(5)
    sw, sh = 48, 40
    re, im = rng.standard_normal((2, sh * sw)).astype(np.float32)
    s = O.CtfStrip(sw=sw, sh=sh, pixel_a=2.0, wavelength=0.0197, cs_a=2.7e7, amp_contrast=0.07,
                   cuton_freq=0.02, defocus1=-25000.0, defocus2=-25000.0, astig_angle_rad=0.0,
                   has_astigmatism=0, plate_phase_rad=0.0, tilt_axis_rad=0.0)
    r1, i1 = O.ctf_correct_strip(re, im, s)
    r2, i2 = O.ctf_correct_strip(r1, i1, s)
    np.testing.assert_array_equal(r2, re)
    np.testing.assert_array_equal(i2, im)
    assert r1[0] == re[0]  # DC is below the cut-on frequency
    flipped = r1 != re
    assert 0.05 < flipped.mean() < 0.95
    np.testing.assert_array_equal(r1[flipped], -re[flipped])
