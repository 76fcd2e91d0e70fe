"""Known-answer tests that pin the CPU oracle (oracle/tilt_oracle.cpp).

The reference ships no tests for its reconstruction arithmetic, so the oracle
is pinned here against analytic answers: FFT vs numpy, the R-weighting of a
delta row, zero response to a constant row, plain smearing at 0 degrees, the
fill rules at out-of-range samples, the adjoint identity between back- and
forward projection, point-source geometry, and the reference's panic on short
tilt files.
"""
import numpy as np
import pytest

import oracle as O
from tgutil import rel_l2, random_stack, smooth_stack, angles


@pytest.mark.parametrize("n", [2, 8, 12, 30, 97, 384, 500, 512, 1024])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    assert rel_l2(O.fft(x, precision=64), ref) < 1e-13
    assert rel_l2(O.fft(x, inverse=True, precision=64), np.fft.ifft(x) * n) < 1e-13
    assert rel_l2(O.fft(x, precision=32), ref) < 5e-7


def test_weight_table_formula():
    # apps/tilt/src/main.rs:349-369 restated in numpy float32
    n, c, f = 64, np.float32(0.35), np.float32(0.05)
    fb = np.minimum(np.arange(n), n - np.arange(n)).astype(np.float32)
    w = fb / np.float32(n // 2 + 1)
    d = w - c
    exp = np.where(w <= c, w, w * np.exp((-d * d) / (np.float32(2.0) * f * f)).astype(np.float32))
    got = O.weight_table(n, 0.35, 0.05)
    assert got[0] == 0.0  # DC removed
    np.testing.assert_allclose(got, exp, rtol=2e-7, atol=0)
    # exact filter size and Hamming window
    got = O.weight_table(n, 0.3, 0.05, exact_filter_size=40, hamming=True)
    w = fb / np.float32(40)
    h = np.where(w <= np.float32(0.3), np.float32(0.54) + np.float32(0.46) *
                 np.cos(np.float32(np.pi) * w / np.float32(0.3)), np.float32(0.0))
    np.testing.assert_allclose(got, w * h, rtol=2e-6, atol=1e-7)


def test_rweight_delta_row_is_inverse_transform_of_weights():
    n = 48
    row = np.zeros((1, n))
    row[0, 0] = 1.0
    got = O.rweight(row, 0.35, 0.05, precision=64)[0]
    w = O.weight_table(n, 0.35, 0.05, precision=64)
    np.testing.assert_allclose(got, np.real(np.fft.ifft(w)), atol=1e-14)


def test_rweight_constant_row_vanishes():
    rows = np.full((3, 128), 7.25, np.float32)
    assert np.max(np.abs(O.rweight(rows, 0.35, 0.05))) < 1e-5


def test_zero_degree_single_view_smears():
    nx, ny = 16, 3
    proj = random_stack(1, ny, nx, seed=1)
    p = O.Params(nx, ny, 1, [0.0], thickness=5, no_weight=True, no_cosine_stretch=True)
    vol, _ = O.run(p, proj, 32)
    mean = np.float32(proj.astype(np.float64).mean())
    for iy in range(ny):
        for oz in range(5):
            np.testing.assert_array_equal(vol[iy, oz, :nx - 1], proj[0, iy, :nx - 1])
            assert vol[iy, oz, nx - 1] == mean  # x0 = nx-1 is out of range: mean fill


@pytest.mark.parametrize("fill", ["mean", "zero", "edge"])
def test_fill_modes_out_of_range(fill):
    nx, ny, onx = 8, 2, 12
    proj = random_stack(1, ny, nx, seed=2)
    p = O.Params(nx, ny, 1, [0.0], width=onx, thickness=1, no_weight=True,
                 no_cosine_stretch=True, fill_mode=fill)
    vol, _ = O.run(p, proj, 32)
    mean = np.float32(proj.astype(np.float64).mean())
    for iy in range(ny):
        row = proj[0, iy]
        for ox in range(onx):
            x0 = ox - 6 + 4
            if 0 <= x0 <= nx - 2:
                assert vol[iy, 0, ox] == row[x0]
            else:
                want = {"mean": mean, "zero": 0.0,
                        "edge": row[0] if x0 < 0 else row[nx - 1]}[fill]
                assert vol[iy, 0, ox] == np.float32(want)


def test_adjoint_identity():
    # forward_project is the exact transpose of the zero-fill back-projector
    # without the 1/N factor (main.rs:756-896), including the x-tilt split
    nx, ny, nz = 24, 10, 7
    ang = np.linspace(-50, 50, nz).astype(np.float32)
    p = O.Params(nx, ny, nz, ang, thickness=9, width=20, xtilt=np.full(nz, 4.0),
                 fill_mode="zero", no_weight=True, no_cosine_stretch=True)
    rng = np.random.default_rng(3)
    proj = rng.standard_normal((nz, ny, nx))
    vol = rng.standard_normal((ny, 9, 20))
    bp = O.backproject(p, proj, np.zeros(nz), precision=64)
    fp = O.forward_project(p, vol, precision=64)
    lhs = np.vdot(bp, vol) * nz
    rhs = np.vdot(proj, fp)
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs)


def test_point_source_reconstructs_at_its_voxel():
    nx, ny, nz, onz = 64, 2, 61, 32
    ang = angles(-60, 60, 2)
    ox0, oz0 = 40, 11
    proj = np.zeros((nz, ny, nx), np.float32)
    xs = np.arange(nx)
    for v, a in enumerate(ang):
        t = np.deg2rad(np.float64(a))
        xc = (ox0 - nx / 2) * np.cos(t) + (oz0 - onz / 2) * np.sin(t) + nx / 2
        proj[v, :, :] = np.exp(-0.5 * ((xs - xc) / 0.8) ** 2)
    # cosine stretch is left off: the reference stretches the data AND keeps
    # cos(t) in the back-projector (main.rs:446-488 with 1021), which moves
    # off-axis points; the geometry alone is checked here.
    p = O.Params(nx, ny, nz, ang, thickness=onz, radial=(0.35, 0.05), fill_mode="zero",
                 no_cosine_stretch=True)
    vol, _ = O.run(p, proj, 64)
    oz, ox = np.unravel_index(np.argmax(vol[0]), vol[0].shape)
    assert (ox, oz) == (ox0, oz0)


def test_short_tilt_file():
    nx, ny, nz = 16, 4, 5
    proj = random_stack(nz, ny, nx, seed=4)
    ang = np.array([-20, -10, 0], np.float32)  # fewer angles than sections
    with pytest.raises(RuntimeError):  # apply_cosine_stretch indexes out of bounds
        O.run(O.Params(nx, ny, nz, ang, thickness=6), proj, 32)
    # without stretch: 3 views back-projected, still scaled by 1/nz (main.rs:685,705)
    p = O.Params(nx, ny, nz, ang, thickness=6, no_cosine_stretch=True, no_weight=True)
    vol, _ = O.run(p, proj, 64)
    p3 = O.Params(nx, ny, 3, ang, thickness=6, no_cosine_stretch=True, no_weight=True)
    means = np.array([proj[v].astype(np.float64).mean() for v in range(3)])
    v3 = O.backproject(p3, proj[:3].astype(np.float64), means, precision=64)
    np.testing.assert_allclose(vol, v3 * 3 / 5, rtol=1e-12, atol=1e-12)


def test_ref32_close_to_geometry_matched_ref64():
    nx, ny, nz = 96, 6, 31
    proj = smooth_stack(nz, ny, nx, seed=5)
    p = O.Params(nx, ny, nz, angles(-60, 60, 4), thickness=40, radial=(0.35, 0.035))
    v32, s32 = O.run(p, proj, 32)
    v64, s64 = O.run(p, proj, "64g")
    assert rel_l2(v32, v64) < 1e-5
    assert abs(s32["amean"] - s64["amean"]) <= 1e-5 * max(1e-3, abs(s64["amean"]))


def test_lowpass_kat():
    v = np.full((4, 5, 6), 2.5, np.float32)
    np.testing.assert_allclose(O.lowpass(v), v, rtol=1e-6)
    d = np.zeros((5, 5, 5), np.float64)
    d[2, 2, 2] = 27.0
    out = O.lowpass(d, precision=64)
    np.testing.assert_allclose(out[1:4, 1:4, 1:4], np.ones((3, 3, 3)), atol=1e-12)
    assert abs(out.sum() - 27.0) < 1e-9


def test_output_stats_rule():
    rng = np.random.default_rng(6)
    v = rng.standard_normal((5, 7, 9)).astype(np.float32)
    out, st = O.output_stats(v, densweight=2.0, outscale=0.5, outadd=1.0)
    want = (v * np.float32(2.0)) * np.float32(0.5) + np.float32(1.0)
    np.testing.assert_array_equal(out, want)
    smeans = [np.float32(s.astype(np.float64).mean()) for s in want]
    gmean = np.float32(sum(np.float64(m) * 63 for m in smeans) / (63 * 5))
    assert st["amin"] == want.min() and st["amax"] == want.max() and st["amean"] == gmean


def test_cubic_stretch_identity_at_zero_degrees():
    proj = random_stack(1, 3, 20, seed=7)
    out = O.cosine_stretch(proj, [0.0], cubic=True)
    np.testing.assert_array_equal(out, proj)


def test_linear_stretch_formula():
    nx = 32
    proj = random_stack(1, 1, nx, seed=8)
    out = O.cosine_stretch(proj, [40.0])[0, 0]
    rad = np.float32(40.0) * np.float32(np.pi) / np.float32(180.0)
    s = np.float32(1.0) / np.float32(np.cos(np.float64(rad)))
    c = np.float32(nx / 2)
    for ox in range(nx):
        src = (np.float32(ox) - c) * s + c
        x0 = int(np.floor(src))
        if 0 <= x0 < nx - 1:
            f = src - np.float32(x0)
            want = proj[0, 0, x0] * (np.float32(1) - f) + proj[0, 0, x0 + 1] * f
        elif x0 == nx - 1:
            want = proj[0, 0, x0]
        else:
            want = 0.0
        assert abs(out[ox] - want) <= 2e-7 * max(1.0, abs(want))


@pytest.mark.parametrize("precision", [32, "64g"])
def test_wbp_rows_equals_whole_run_slices(precision):
    # the row-subset flow (means over whole views, only the band rows filtered) gives
    # the same slices as the whole-volume run, in both the f32 and the FP64 forms
    nz, ny, nx = 9, 12, 48
    proj = (smooth_stack(nz, ny, nx, seed=9) * 100.0 + 1000.0).astype(np.float32)
    ang = angles(-48, 48, 12)
    p = O.Params(nx, ny, nz, ang, thickness=20, radial=(0.35, 0.035), log=True)
    whole, _ = O.run(p, proj, precision)
    rows = O.wbp_rows(p, proj, 3, 8, nthreads=4, precision=precision)
    np.testing.assert_array_equal(rows, whole[3:8])


def test_studio_step_is_tilt_with_its_options():
    # imod-studio's reconstruction step (apps/imod-studio/src/main.rs:725-776) is the
    # tilt path with --no-weight --no-cosine-stretch --fill-mode zero and thickness = width:
    # the same positions, lerp, skipped out-of-row samples (zero fill adds +0) and 1/nz
    nz, ny, nx = 11, 5, 40
    proj = random_stack(nz, ny, nx, seed=12, offset=-0.5)
    ang = np.linspace(-55, 55, nz).astype(np.float32)
    studio = O.studio_reconstruct(proj, ang)
    p = O.Params(nx, ny, nz, ang, thickness=nx, no_weight=True, no_cosine_stretch=True, fill_mode="zero")
    tilt, _ = O.run(p, proj, 32)
    np.testing.assert_array_equal(studio, tilt)
    # fewer angles than sections: the loop stops at the last angle, 1/nz still uses the sections
    studio2 = O.studio_reconstruct(proj, ang[:7])
    tilt2, _ = O.run(O.Params(nx, ny, nz, ang[:7], thickness=nx, no_weight=True, no_cosine_stretch=True,
                              fill_mode="zero"), proj, 32)
    np.testing.assert_array_equal(studio2, tilt2)


def test_min_max_mean_matches_the_reference_unit_test():
    # crates/imod-math/src/tests.rs test_min_max_mean (vector in tests/golden): the per-view
    # mean fill (main.rs:616-623) and the output header statistics (main.rs:1077-1093)
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))["min_max_mean"]
    data = np.array(g["data"], np.float32)
    mean = g["mean_num"] / g["mean_den"]
    m = O.view_means(data.reshape(1, 1, -1))
    assert abs(float(m[0]) - mean) < g["tol"]
    _, st = O.output_stats(data.reshape(1, 1, -1))
    assert st["amin"] == g["min"] and st["amax"] == g["max"]
    assert abs(st["amean"] - mean) < g["tol"]
