"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Tolerances (the FP32 one is the bound set for the FP32 path):
  * back-projection alone (no R-weighting, no stretch), FP32 storage: bit-exact
    against ref32 -- sample positions, fill rules, interpolation and the
    per-view accumulation order all follow the reference's f32 operations;
  * whole path with R-weighting, FP32: rel-L2 <= 1e-5 against ref32 (the two
    FFTs round differently);
  * FP16 / BF16 staging: rel-L2 <= 2e-3 against ref64g (FP64 data path with the
    reference's sampling geometry).
"""
import numpy as np
import pytest

import oracle as O
import tiltgpu as T
from tgutil import angles, max_abs, random_stack, rel_l2, smooth_stack

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-5
TOL_HALF = 2e-3


def both(proj, ang, precision=32, storage="fp32", **kw):
    nz, ny, nx = proj.shape
    gkw = dict(kw)
    okw = dict(kw)
    if "gpu" in okw:
        okw["gpu_compat"] = okw.pop("gpu")
    okw.pop("exact_xtilt", None)  # a GPU-side choice of summation order
    vol, st = T.reconstruct(proj, ang, storage=storage, **gkw)
    ref, rst = O.run(O.Params(nx, ny, nz, ang, **okw), proj, precision)
    return vol, st, ref, rst


@pytest.mark.parametrize("fill", ["mean", "zero", "edge"])
@pytest.mark.parametrize("shape", [(21, 9, 64, 64, 40), (15, 10, 48, 60, 33)])
def test_backprojection_bit_exact_fast(fill, shape):
    nz, ny, nx, onx, onz = shape
    proj = random_stack(nz, ny, nx, seed=nx + ny)
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    vol, st, ref, rst = both(proj, ang, no_weight=True, no_cosine_stretch=True, fill_mode=fill,
                             width=onx, thickness=onz)
    np.testing.assert_array_equal(vol, ref)
    assert st["amin"] == rst["amin"] and st["amax"] == rst["amax"]
    assert abs(st["amean"] - rst["amean"]) <= 1e-6 * abs(rst["amean"])


def test_backprojection_bit_exact_zfactor_and_transform():
    nz, ny, nx = 11, 8, 40
    proj = random_stack(nz, ny, nx, seed=3)
    ang = np.linspace(-45, 45, nz).astype(np.float32)
    zf = np.linspace(0.8, 1.3, nz).astype(np.float32)
    vol, _, ref, _ = both(proj, ang, no_weight=True, no_cosine_stretch=True, zfactor=zf,
                          thickness=30, densweight=1.5, outscale=2.0, outadd=-0.25)
    np.testing.assert_array_equal(vol, ref)


def test_backprojection_bit_exact_general_xtilt():
    nz, ny, nx = 13, 12, 48
    proj = random_stack(nz, ny, nx, seed=4)
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    vol, _, ref, _ = both(proj, ang, no_weight=True, no_cosine_stretch=True,
                          xtilt=np.full(nz, 1.5, np.float32), thickness=36, exact_xtilt=True)
    np.testing.assert_array_equal(vol, ref)


@pytest.mark.parametrize("fill", ["mean", "zero", "edge"])
@pytest.mark.parametrize("xt,shape", [(1.5, (15, 21, 70, 75, 37)), (-8.0, (11, 17, 48, 64, 20)),
                                      ("mixed", (13, 9, 40, 33, 50))])
def test_backprojection_bit_exact_xtilt_staged(fill, xt, shape):
    # x-tilt back-projection from staged rows: every row pair, edge row and fill
    # rule as the reference's f32 arithmetic, ragged tiles in x, z and y
    nz, ny, nx, onx, onz = shape
    proj = random_stack(nz, ny, nx, seed=nx + onz)
    ang = np.linspace(-62, 58, nz).astype(np.float32)
    if xt == "mixed":
        xtv = np.linspace(-3.0, 5.0, nz).astype(np.float32)
        xtv[2] = 0.0
        zf = np.linspace(0.9, 1.2, nz).astype(np.float32)
    else:
        xtv, zf = np.full(nz, xt, np.float32), None
    vol, st, ref, rst = both(proj, ang, no_weight=True, no_cosine_stretch=True, fill_mode=fill,
                             xtilt=xtv, zfactor=zf, width=onx, thickness=onz, exact_xtilt=True)
    np.testing.assert_array_equal(vol, ref)
    assert st["amin"] == rst["amin"] and st["amax"] == rst["amax"]


@pytest.mark.parametrize("fill", ["mean", "zero", "edge"])
@pytest.mark.parametrize("xt,shape,zf", [(1.5, (15, 21, 70, 75, 37), False), (-8.0, (11, 17, 48, 64, 20), True),
                                         (0.3, (9, 40, 64, 64, 16), False), (12.0, (7, 9, 40, 33, 50), False)])
def test_backprojection_xtilt_row_sums(fill, xt, shape, zf):
    # one x-tilt for all views: the fast kernel sums every projection row over the
    # views, then each voxel blends its two rows (same rows, fractions, one-row
    # edges and fills as the reference; only the f32 summation order differs)
    nz, ny, nx, onx, onz = shape
    proj = random_stack(nz, ny, nx, seed=nx + onz + 1)
    ang = np.linspace(-62, 58, nz).astype(np.float32)
    zfv = np.linspace(0.9, 1.2, nz).astype(np.float32) if zf else None
    kw = dict(no_weight=True, no_cosine_stretch=True, fill_mode=fill, xtilt=np.full(nz, xt, np.float32),
              zfactor=zfv, width=onx, thickness=onz)
    with T.Session(nx, ny, nz, ang, **kw) as s:
        info = s.kernel_info()
    assert info["xtilt_split"], info
    vol, st, ref, rst = both(proj, ang, **kw)
    assert rel_l2(vol, ref) <= 1e-6
    assert np.abs(vol - ref).max() <= 1e-5 * max(1.0, float(np.abs(ref).max()))
    assert abs(st["amin"] - rst["amin"]) <= 1e-5 and abs(st["amax"] - rst["amax"]) <= 1e-5
    exact, _, _, _ = both(proj, ang, exact_xtilt=True, **kw)
    np.testing.assert_array_equal(exact, ref)


def test_backprojection_bit_exact_local_alignment():
    nz, ny, nx = 9, 16, 40
    proj = random_stack(nz, ny, nx, seed=5)
    ang = np.linspace(-40, 40, nz).astype(np.float32)
    rng = np.random.default_rng(5)
    rows = []
    for v in range(nz):
        for x in (5.0, 20.0, 35.0):
            for y in (2.0, 8.0, 14.0):
                rows.append([v, x, y, rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0)])
    local = np.array(rows, np.float32)
    vol, _, ref, _ = both(proj, ang, no_weight=True, no_cosine_stretch=True, local=local,
                          thickness=24)
    np.testing.assert_array_equal(vol, ref)


@pytest.mark.parametrize("nx", [64, 96, 100, 98, 97])
def test_whole_path_fp32(nx):
    nz, ny = 19, 6
    proj = smooth_stack(nz, ny, nx, seed=nx)
    ang = angles(-54, 54, 6)
    vol, st, ref, rst = both(proj, ang, radial=(0.35, 0.035), thickness=30)
    assert rel_l2(vol, ref) <= TOL_FP32
    assert abs(st["amean"] - rst["amean"]) <= 1e-4 * max(abs(rst["amean"]), 1e-3)


def _local_rows(nz, nx, ny, seed, skip=()):
    rng = np.random.default_rng(seed)
    rows = []
    for v in range(nz):
        if v in skip:  # a view without patches: no correction, still the two-row split
            continue
        for x in np.linspace(4, nx - 5, 3):
            for y in np.linspace(2, ny - 3, 3):
                rows.append([v, x, y, rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0)])
    return np.array(rows, np.float32)


@pytest.mark.parametrize("ny,xt", [(16, 0.0), (13, 1.5)])
def test_sirt_local_alignment_vs_oracle(ny, xt):
    # local corrections from the per-session table, in the back-projector (bit-exact
    # alone) and in the multi-row reprojector (summation order differs: tolerance)
    nz, nx = 11, 44
    proj = random_stack(nz, ny, nx, seed=80 + ny)
    ang = angles(-50, 50, 10)
    kw = dict(sirt=2, sirt_relax=0.9, no_weight=True, no_cosine_stretch=True, thickness=20,
              local=_local_rows(nz, nx, ny, seed=ny, skip=(3,)))
    if xt:
        kw["xtilt"] = np.full(nz, xt, np.float32)
    vol, _, ref, _ = both(proj, ang, **kw)
    assert rel_l2(vol, ref) <= 1e-6
    vol, _, ref, _ = both(smooth_stack(nz, ny, nx, seed=81), ang, sirt=2, radial=(0.35, 0.035),
                          thickness=20, local=kw["local"])
    assert rel_l2(vol, ref) <= TOL_FP32


@pytest.mark.parametrize("nx,opts", [(256, dict()), (1024, dict(cosine_interp="cubic")),
                                     (384, dict()), (768, dict(fill_mode="edge", sirt=1)),
                                     (512, dict(fill_mode="edge", max_cosine_tilt=40.0)),
                                     (256, dict(fill_mode="zero", xtilt=1.0)),
                                     (256, dict(sirt=2, sirt_relax=0.8))])
def test_whole_path_fp32_radix8_rows(nx, opts):
    # 2^k and 3*2^k rows take the register-resident FFT; rows of both parities, fills,
    # stretch, SINGLE staging (x-tilt) and the SIRT residual
    nz, ny = 9, 5
    proj = smooth_stack(nz, ny, nx, seed=nx + ny)
    ang = angles(-56, 56, 14)
    kw = dict(opts)
    if "xtilt" in kw:
        kw["xtilt"] = np.full(nz, kw["xtilt"], np.float32)
    vol, _, ref, _ = both(proj, ang, radial=(0.35, 0.035), thickness=24, **kw)
    assert rel_l2(vol, ref) <= TOL_FP32


@pytest.mark.parametrize("opts", [dict(cosine_interp="cubic"), dict(hamming=True, radial=(0.3, 0.0)),
                                  dict(exact_filter_size=40), dict(log=True),
                                  dict(max_cosine_tilt=30.0, fill_mode="edge"),
                                  dict(width=80, thickness=17)])
def test_whole_path_options(opts):
    nz, ny, nx = 17, 6, 64
    proj = smooth_stack(nz, ny, nx, seed=11)
    ang = angles(-48, 48, 6)
    vol, _, ref, _ = both(proj, ang, **opts)
    assert rel_l2(vol, ref) <= TOL_FP32


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
def test_half_storage_vs_fp64(storage):
    nz, ny, nx = 31, 8, 128
    proj = smooth_stack(nz, ny, nx, seed=21)
    ang = angles(-60, 60, 4)
    vol, _, ref, _ = both(proj, ang, precision="64g", storage=storage, radial=(0.35, 0.035),
                          thickness=48)
    err = rel_l2(vol, ref)
    assert err <= (TOL_HALF if storage == "fp16" else 4 * TOL_HALF), err


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
@pytest.mark.parametrize("xt", [0.0, 2.0])
def test_sirt_half_storage_vs_fp64(storage, xt):
    # half staging forms also reproject from a scaled FP16 copy of the volume (with one
    # x-tilt for all views: of its blended rows)
    nz, ny, nx = 31, 19, 96
    proj = smooth_stack(nz, ny, nx, seed=22)
    ang = angles(-60, 60, 4)
    kw = dict(xtilt=np.full(nz, xt, np.float32)) if xt else {}
    vol, _, ref, _ = both(proj, ang, precision="64g", storage=storage, radial=(0.35, 0.035),
                          thickness=40, sirt=4, sirt_relax=0.8, **kw)
    err = rel_l2(vol, ref)
    assert err <= (TOL_HALF if storage == "fp16" else 4 * TOL_HALF), err


def test_sirt_no_xtilt():
    nz, ny, nx = 15, 6, 48
    proj = smooth_stack(nz, ny, nx, seed=31)
    ang = angles(-56, 56, 8)
    vol, _, ref, _ = both(proj, ang, sirt=3, sirt_relax=0.7, thickness=24)
    assert rel_l2(vol, ref) <= TOL_FP32


def test_sirt_bit_exact_without_filter():
    # no R-weighting, no stretch: back-projection, reprojection (per-bin order of the
    # reference's serial splat), residual and update are all exact f32 operations
    nz, ny, nx = 13, 11, 40
    proj = random_stack(nz, ny, nx, seed=30)
    ang = angles(-60, 60, 10)
    vol, _, ref, _ = both(proj, ang, sirt=2, sirt_relax=0.8, no_weight=True, no_cosine_stretch=True,
                          thickness=22, width=44)
    np.testing.assert_array_equal(vol, ref)


@pytest.mark.parametrize("ny", [10, 17])
def test_sirt_xtilt_rows_and_edges(ny):
    # x-tilt reprojection: rows shift by dx*sin(x-tilt) and split in two; edge rows
    # take the reference's one-row branch; views with zero x-tilt stay one-row
    nz, nx = 12, 48
    proj = random_stack(nz, ny, nx, seed=40 + ny)
    ang = angles(-55, 55, 10)
    xt = np.linspace(-4.0, 4.0, nz).astype(np.float32)
    xt[3] = 0.0
    vol, _, ref, _ = both(proj, ang, sirt=2, sirt_relax=0.9, no_weight=True, no_cosine_stretch=True,
                          xtilt=xt, thickness=20, width=52)
    assert rel_l2(vol, ref) <= 1e-6


@pytest.mark.parametrize("ny,xt", [(10, -3.0), (17, 2.0), (24, 6.5), (33, 0.7)])
def test_sirt_common_xtilt_blended_copy(ny, xt, monkeypatch):
    # one x-tilt for every view: the reprojector projects a copy whose rows are the
    # reference's two-slice blends (edge rows, raised floors), summed in another order
    nz, nx = 12, 56
    proj = random_stack(nz, ny, nx, seed=50 + ny)
    ang = angles(-55, 55, 10)
    kw = dict(sirt=2, sirt_relax=0.9, no_weight=True, no_cosine_stretch=True,
              xtilt=np.full(nz, xt, np.float32), thickness=22, width=60)
    vol, _, ref, _ = both(proj, ang, **kw)
    assert rel_l2(vol, ref) <= 1e-6
    monkeypatch.setenv("TG_FP_VARIANT", "0")  # no copy: slices read from the volume itself
    direct, _ = T.reconstruct(proj, ang, **kw)
    assert rel_l2(vol, direct) <= 1e-6


@pytest.mark.parametrize("xt", [0.0, 1.5])
def test_sirt_thick_many_views_vs_oracle(xt):
    # a thick volume and 61 views over 8 iterations: the size where the reference's
    # un-normalised SIRT update grows fastest; the GPU must follow the oracle there too
    ang = angles(-60, 60, 2)
    nz, ny, nx = len(ang), 6, 512
    proj = (smooth_stack(nz, ny, nx, seed=71) * 300.0 + 20000.0).astype(np.float32)
    kw = dict(sirt=8, log=True, radial=(0.35, 0.035), thickness=300)
    if xt:
        kw["xtilt"] = np.full(nz, xt, np.float32)
    vol, st, ref, rst = both(proj, ang, **kw)
    assert np.isfinite(vol).all()
    assert rel_l2(vol, ref) <= TOL_FP32, (rel_l2(vol, ref), float(np.abs(ref).max()))


def test_sirt_xtilt_log_fake():
    nz, ny, nx = 11, 10, 40
    proj = (smooth_stack(nz, ny, nx, seed=32) * 1000.0).astype(np.float32)
    ang = angles(-50, 50, 10)
    vol, _, ref, _ = both(proj, ang, sirt=2, log=True, xtilt=np.full(nz, 1.5, np.float32),
                          thickness=20, fake_sirt=1)
    assert rel_l2(vol, ref) <= TOL_FP32


def test_fake_sirt_wbp():
    nz, ny, nx = 13, 7, 32
    proj = smooth_stack(nz, ny, nx, seed=33)
    vol, _, ref, _ = both(proj, angles(-48, 48, 8), fake_sirt=2, thickness=16)
    assert rel_l2(vol, ref) <= TOL_FP32


def test_gpu_compat_mode():
    nz, ny, nx = 15, 6, 48
    proj = smooth_stack(nz, ny, nx, seed=34)
    ang = angles(-56, 56, 8)
    vol, _, ref, _ = both(proj, ang, gpu=True, thickness=20, sirt=2,
                          xtilt=np.full(nz, 2.0, np.float32))
    assert rel_l2(vol, ref) <= TOL_FP32


def test_reference_gpu_seam_bit_exact():
    # GpuSession::new + reconstruct_row on already-filtered data (gpu.rs:43-269)
    nz, ny, nx, onx, onz = 9, 5, 40, 44, 21
    proj = random_stack(nz, ny, nx, seed=35)
    ang = np.linspace(-50, 50, nz).astype(np.float32)
    rad = ang * np.float32(np.pi) / np.float32(180.0)
    cs = np.stack([np.cos(rad.astype(np.float64)), np.sin(rad.astype(np.float64))], 1).astype(np.float32)
    p = O.Params(nx, ny, nz, ang, width=onx, thickness=onz, gpu_compat=True)
    ref = O.backproject(p, proj, np.zeros(nz, np.float32))
    g = T.GpuSession(proj, cs, nx, ny, nz, onx, onz)
    for iy in (0, 2, 4):
        np.testing.assert_array_equal(g.reconstruct_row(iy), ref[iy])
    g.close()


def test_apply_rweighting_stage():
    proj = smooth_stack(3, 4, 100, seed=36)
    got = T.apply_rweighting(proj, 0.35, 0.05)
    want = O.rweight(proj, 0.35, 0.05)
    assert rel_l2(got, want) <= 1e-6


def test_deterministic_and_resident():
    nz, ny, nx = 21, 16, 96
    proj = smooth_stack(nz, ny, nx, seed=37)
    ang = angles(-60, 60, 6)
    with T.Session(nx, ny, nz, ang, thickness=40, storage="fp16") as s:
        s.upload(proj)
        s.reconstruct()
        a, sa = s.download()
        s.reconstruct()  # projections stay resident; log is not applied twice
        b, sb = s.download()
    np.testing.assert_array_equal(a, b)
    assert sa == sb


def test_short_tilt_file_errors():
    nz, ny, nx = 6, 4, 32
    proj = random_stack(nz, ny, nx, seed=38)
    ang = np.array([-10, 0, 10], np.float32)
    with pytest.raises(T.TiltGpuError) as e:
        T.reconstruct(proj, ang)
    assert e.value.code == -8
    vol, _, ref, _ = both(proj, ang, no_cosine_stretch=True, thickness=10)
    assert rel_l2(vol, ref) <= TOL_FP32


def test_synthetic_phantom_is_seeded():
    ang = angles(-60, 60, 10)
    a = T.synth_projections(ang, nx=96, ny=16, vol_nz=40, n_ell=30, rmax=10, n_beads=4, seed=7)
    b = T.synth_projections(ang, nx=96, ny=16, vol_nz=40, n_ell=30, rmax=10, n_beads=4, seed=7)
    c = T.synth_projections(ang, nx=96, ny=16, vol_nz=40, n_ell=30, rmax=10, n_beads=4, seed=8)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert np.isfinite(a).all()


def test_c1_size_subset_and_linearity():
    # config-1 geometry (61 views, 512^2 -> 512x512x200): the oracle checks a
    # subset of slices (FP16 against the FP64 oracle: test_gpu_parity_configs.py)
    ang = angles(-60, 60, 2)
    nx = ny = 512
    proj = T.synth_projections(ang, nx=nx, ny=ny, vol_nz=200, n_ell=300, rmin=3, rmax=40,
                               dmin=0.2, dmax=1.0, n_beads=40, bead_r=5, bead_d=5.0,
                               noise_kind=1, noise=0.5, seed=1)
    kw = dict(radial=(0.35, 0.035), thickness=200)
    v32, s32 = T.reconstruct(proj, ang, storage="fp32", **kw)
    p = O.Params(nx, ny, len(ang), ang, **kw)
    ys = (0, 8)
    ref = O.wbp_rows(p, proj, *ys)
    out, _ = O.output_stats(ref)
    assert rel_l2(v32[ys[0]:ys[1]], out) <= TOL_FP32
    # linearity of the whole path in the projections (size-independent property)
    v2, _ = T.reconstruct((2.0 * proj).astype(np.float32), ang, storage="fp32", **kw)
    assert rel_l2(v2, 2.0 * v32) <= 1e-6
