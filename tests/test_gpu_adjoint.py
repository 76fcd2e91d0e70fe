"""The device reprojector is the transpose of the device back-projector (the
reference's forward_project is exactly the transpose of its back-projection
without the fill and the 1/N, apps/tilt/src/main.rs:831-896 vs 1002-1090), checked
through the public SIRT-in-steps entry points: with all projections zero and no
R-weighting, one SIRT iteration at relaxation 1 maps a restored volume v to
v - BP(FP v) (the residual -FP v, its mean fill 0), so M v = BP(FP v) comes out
of the device for any v, and M must be symmetric: <u, M v> = <M u, v>.  A lost or
doubled write in either kernel breaks the symmetry (the check on write races that
a sanitizer would make)."""
import numpy as np
import pytest

import tiltgpu as T
from tgutil import angles

pytestmark = pytest.mark.gpu


def apply_m(nx, ny, nz, ang, vol, **kw):
    with T.Session(nx, ny, nz, ang, sirt=1, sirt_relax=1.0, no_weight=True, fill_mode="zero", **kw) as s:
        s.upload(np.zeros((nz, ny, nx), np.float32))
        s.sirt_restore(vol, 0)
        s.sirt_iterate(1)
        after, _ = s.sirt_save()
    return vol.astype(np.float64) - after.astype(np.float64)


@pytest.mark.parametrize("kw,tol", [(dict(storage="fp32"), 2e-6),
                                    (dict(storage="fp32", xtilt=1.5), 2e-6),
                                    (dict(storage="fp16"), 3e-3)])
def test_reprojection_is_the_transpose_of_backprojection(kw, tol):
    nz, ny, nx, thick = 17, 24, 96, 40
    ang = angles(-56, 56, 7)
    opts = dict(thickness=thick, **{k: v for k, v in kw.items() if k != "xtilt"})
    if "xtilt" in kw:
        opts["xtilt"] = np.full(nz, kw["xtilt"], np.float32)
    rng = np.random.default_rng(4)
    u = rng.standard_normal((ny, thick, nx)).astype(np.float32)
    v = rng.standard_normal((ny, thick, nx)).astype(np.float32)
    mu = apply_m(nx, ny, nz, ang, u, **opts)
    mv = apply_m(nx, ny, nz, ang, v, **opts)
    a = float(np.vdot(u.astype(np.float64), mv))
    b = float(np.vdot(mu, v.astype(np.float64)))
    scale = np.linalg.norm(u) * np.linalg.norm(mv)
    assert abs(a - b) <= tol * scale, (a, b, scale)
    # M is positive semidefinite: <v, M v> = |FP v|^2 / N >= 0, and not zero here
    assert float(np.vdot(v.astype(np.float64), mv)) > 0.0
