"""GPU parity at the geometries of the benchmark configurations.

The small parity cases elsewhere are at most 128 columns wide.  These run the
CUDA path through the C ABI at full width, on strips of rows that the CPU
oracle finishes in seconds:

  * SIRT with a shared x-tilt (61 views at +-60 deg in 2 deg steps, 1024 wide,
    thickness 400, x-tilt 1.5 deg, Poisson counts with --log): the x-tilt band
    reaches +-13 rows there, so the row-sum back-projection, the blended-row
    reprojection copy and their edge rules all work where they matter most;
  * large plain WBP (121 jittered views, 2048 wide, thickness 800);
  * FP16 staging checked against the FP64 oracle (ref64g), not against the
    GPU's own FP32 output.

Tolerances: FP32 rel-L2 <= 1e-5 against ref32; FP16 <= 2e-3 and BF16 <= 8e-3
against ref64g (FP64 data path with the reference's f32 sampling geometry).
Values the FP16 staging cannot hold are reported as TG_ERR_RANGE.
"""
import numpy as np
import pytest

import oracle as O
import tiltgpu as T
from tgutil import angles, rel_l2, smooth_stack

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5
TOL = {"fp16": 2e-3, "bf16": 8e-3}


# ---- SIRT with x-tilt at the 1024-wide, 400-thick, 61-view geometry ----
C3_ROWS = 24


@pytest.fixture(scope="module")
def c3_strip():
    ang = angles(-60, 60, 2)
    nx = 1024
    proj = T.synth_projections(ang, nx=nx, ny=C3_ROWS, vol_nz=400, n_ell=300, rmin=3, rmax=40,
                               dmin=0.2, dmax=1.0, n_beads=40, bead_r=5, bead_d=5.0, noise_kind=2,
                               noise=20000.0, xtilt_deg=1.5, seed=3)
    kw = dict(radial=(0.35, 0.035), thickness=400, log=True, sirt=3, sirt_relax=0.3,
              xtilt=np.full(len(ang), 1.5, np.float32))
    p = O.Params(nx, C3_ROWS, len(ang), ang, **kw)
    ref32, rst = O.run(p, proj, 32)
    ref64, _ = O.run(p, proj, "64g")
    return proj, ang, kw, ref32, rst, ref64


def test_c3_strip_sirt_fp32_vs_oracle(c3_strip):
    proj, ang, kw, ref32, rst, _ = c3_strip
    vol, st = T.reconstruct(proj, ang, storage="fp32", **kw)
    with T.Session(proj.shape[2], proj.shape[1], proj.shape[0], ang, **kw) as s:
        assert s.kernel_info()["xtilt_split"]  # row sums + two-row blend (the default form)
    assert np.isfinite(vol).all()
    assert rel_l2(vol, ref32) <= TOL_FP32, rel_l2(vol, ref32)
    assert st["amin"] == pytest.approx(rst["amin"], rel=1e-5, abs=1e-6)
    assert st["amax"] == pytest.approx(rst["amax"], rel=1e-5, abs=1e-6)


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
def test_c3_strip_sirt_half_vs_fp64(c3_strip, storage):
    proj, ang, kw, _, _, ref64 = c3_strip
    vol, _ = T.reconstruct(proj, ang, storage=storage, **kw)
    err = rel_l2(vol, ref64)
    assert err <= TOL[storage], err


# ---- large plain WBP: 2048 wide, 121 jittered views, thickness 800 ----
@pytest.fixture(scope="module")
def c2_strip():
    rng = np.random.default_rng(2)
    ang = (np.arange(-60, 61, 1.0) + rng.normal(0.0, 0.1, 121)).astype(np.float32)
    nx, ny = 2048, 8
    proj = T.synth_projections(ang, nx=nx, ny=ny, vol_nz=800, n_ell=5000, rmin=3, rmax=40, dmin=0.2,
                               dmax=1.0, n_beads=200, bead_r=5, bead_d=5.0, noise_kind=2, noise=20000.0,
                               seed=1000)
    kw = dict(radial=(0.35, 0.035), thickness=800, log=True)
    p = O.Params(nx, ny, len(ang), ang, **kw)
    ref32, _ = O.run(p, proj, 32)
    ref64, _ = O.run(p, proj, "64g")
    return proj, ang, kw, ref32, ref64


def test_c2_strip_fp32_vs_oracle(c2_strip):
    proj, ang, kw, ref32, _ = c2_strip
    vol, _ = T.reconstruct(proj, ang, storage="fp32", **kw)
    assert rel_l2(vol, ref32) <= TOL_FP32, rel_l2(vol, ref32)


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
def test_c2_strip_half_vs_fp64(c2_strip, storage):
    proj, ang, kw, _, ref64 = c2_strip
    vol, _ = T.reconstruct(proj, ang, storage=storage, **kw)
    err = rel_l2(vol, ref64)
    assert err <= TOL[storage], err


# ---- 512^2 x 61 views -> 512x512x200: FP16 on a slice subset against ref64g ----
def test_c1_slices_fp16_vs_fp64():
    ang = angles(-60, 60, 2)
    nx = ny = 512
    proj = T.synth_projections(ang, nx=nx, ny=ny, vol_nz=200, n_ell=300, rmin=3, rmax=40, dmin=0.2,
                               dmax=1.0, n_beads=40, bead_r=5, bead_d=5.0, noise_kind=1, noise=0.5,
                               seed=1)
    kw = dict(radial=(0.35, 0.035), thickness=200)
    v16, _ = T.reconstruct(proj, ang, storage="fp16", **kw)
    p = O.Params(nx, ny, len(ang), ang, **kw)
    for ys in ((0, 8), (252, 260)):
        ref64 = O.wbp_rows(p, proj, *ys, precision="64g")  # means over whole views
        err = rel_l2(v16[ys[0]:ys[1]], ref64)
        assert err <= TOL["fp16"], (ys, err)


# ---- FP16 range: values the staging cannot hold are an error, not silent infinities ----
def test_fp16_range_reported_for_large_values():
    nz, ny, nx = 15, 6, 64
    proj = (smooth_stack(nz, ny, nx, seed=81) * 4.0e5).astype(np.float32)
    ang = angles(-56, 56, 8)
    kw = dict(radial=(0.35, 0.035), thickness=24)
    with pytest.raises(T.TiltGpuError) as e:
        T.reconstruct(proj, ang, storage="fp16", **kw)
    assert e.value.code == -12
    p = O.Params(nx, ny, nz, ang, **kw)
    ref, _ = O.run(p, proj, 32)
    for storage in ("fp32", "bf16"):  # the f32 range holds these values
        vol, _ = T.reconstruct(proj, ang, storage=storage, **kw)
        assert rel_l2(vol, ref) <= (TOL_FP32 if storage == "fp32" else TOL["bf16"])


def test_fp16_range_reported_for_diverging_sirt():
    # a relaxation far above 1 makes the reference's un-normalised SIRT update grow
    # every iteration; the FP32 form keeps going (finite, like the reference), the
    # FP16 form reports that its residuals left the FP16 range
    nz, ny, nx = 21, 4, 64
    proj = smooth_stack(nz, ny, nx, seed=82)
    ang = angles(-60, 60, 6)
    kw = dict(radial=(0.35, 0.035), thickness=32, sirt=6, sirt_relax=40.0)
    v32, _ = T.reconstruct(proj, ang, storage="fp32", **kw)
    assert np.isfinite(v32).all() and np.abs(v32).max() > 65520.0
    with T.Session(nx, ny, nz, ang, storage="fp16", **kw) as s:
        s.upload(proj)
        with pytest.raises(T.TiltGpuError) as e:
            s.reconstruct()
        assert e.value.code == -12
        # the error word is cleared: the same session runs a converging case afterwards
    ok, _ = T.reconstruct(proj, ang, storage="fp16", radial=(0.35, 0.035), thickness=32, sirt=2,
                          sirt_relax=0.5)
    assert np.isfinite(ok).all()
