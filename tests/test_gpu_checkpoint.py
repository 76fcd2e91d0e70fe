"""SIRT in steps with checkpoints (tg_sirt_*): a run saved after k iterations
and restored into a fresh session continues to tg_reconstruct's n-iteration
result bit for bit (the loop of apps/tilt/src/main.rs:919-975, split between
graph launches)."""
import numpy as np
import pytest

import tiltgpu as T
from tgutil import angles, smooth_stack

pytestmark = pytest.mark.gpu

CASES = [
    dict(storage="fp32"),
    dict(storage="fp16", xtilt=1.5),
    dict(storage="fp32", use_graphs=False, fake_sirt=1),
    dict(storage="bf16", local=True),
]


def series(seed=3):
    nz, ny, nx = 25, 24, 96
    proj = (smooth_stack(nz, ny, nx, seed=seed) * 200.0 + 1000.0).astype(np.float32)
    return proj, angles(-60, 60, 5)  # 25 views


def opts(case, nz):
    kw = dict(thickness=40, radial=(0.35, 0.035), log=True, sirt=6, sirt_relax=0.3)
    kw.update({k: v for k, v in case.items() if k not in ("xtilt", "local")})
    if "xtilt" in case:
        kw["xtilt"] = np.full(nz, case["xtilt"], np.float32)
    if case.get("local"):
        rng = np.random.default_rng(5)
        rows = []
        for v in range(nz):  # 3x3 patches per view: (view, x, y, dx, dy)
            for py in (4.0, 12.0, 20.0):
                for px in (16.0, 48.0, 80.0):
                    rows.append((v, px, py, rng.uniform(-0.8, 0.8), rng.uniform(-0.5, 0.5)))
        kw["local"] = np.array(rows, np.float32)
    return kw


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}={v}" for k, v in c.items()))
@pytest.mark.parametrize("k", [0, 2, 6])
def test_restore_continues_the_run(case, k):
    proj, ang = series()
    nz, ny, nx = proj.shape
    kw = opts(case, nz)
    whole, wst = T.reconstruct(proj, ang, **kw)
    with T.Session(nx, ny, nz, ang, **kw) as s:
        s.upload(proj)
        s.sirt_begin()
        if k:
            s.sirt_iterate(1)
            s.sirt_iterate(k - 1)
        state, done = s.sirt_save()
    assert done == k
    with T.Session(nx, ny, nz, ang, **kw) as s:
        s.upload(proj)
        s.sirt_restore(state, done)
        s.sirt_iterate(6 - k)
        s.sirt_end()
        vol, st = s.download()
        np.testing.assert_array_equal(vol, whole)
        assert (st["amin"], st["amax"], st["amean"]) == (wst["amin"], wst["amax"], wst["amean"])
        # the session then runs tg_reconstruct as usual
        s.reconstruct()
        again, _ = s.download()
        np.testing.assert_array_equal(again, whole)


def test_steps_in_one_session_equal_the_whole_run():
    proj, ang = series(7)
    nz, ny, nx = proj.shape
    kw = opts(dict(storage="fp16"), nz)
    whole, _ = T.reconstruct(proj, ang, **kw)
    with T.Session(nx, ny, nz, ang, **kw) as s:
        s.upload(proj)
        s.sirt_begin()
        for _ in range(3):
            s.sirt_iterate(2)
        s.sirt_end()
        vol, _ = s.download()
    np.testing.assert_array_equal(vol, whole)


def test_out_of_order_calls_are_refused():
    proj, ang = series()
    nz, ny, nx = proj.shape
    kw = opts(dict(storage="fp32"), nz)
    with T.Session(nx, ny, nz, ang, **kw) as s:
        s.upload(proj)
        for bad in (lambda: s.sirt_iterate(1), s.sirt_end, s.sirt_save):
            with pytest.raises(T.TiltGpuError) as e:
                bad()
            assert e.value.code == -1
        s.sirt_begin()
        with pytest.raises(T.TiltGpuError):
            s.sirt_iterate(7)  # beyond sirt_iters
        s.sirt_iterate(6)
        with pytest.raises(T.TiltGpuError):
            s.sirt_iterate(1)
        state, done = s.sirt_save()
        assert done == 6
        with pytest.raises(T.TiltGpuError):
            s.sirt_restore(state, 7)
    kw0 = dict(kw, sirt=0)
    with T.Session(nx, ny, nz, ang, **kw0) as s:
        s.upload(proj)
        with pytest.raises(T.TiltGpuError):
            s.sirt_begin()


def test_output_stage_and_view_mean_match_the_reference_unit_test():
    # crates/imod-math/src/tests.rs test_min_max_mean (vector in tests/golden), through the
    # device: the per-view mean of the uploaded view (tg_session_view_sums) and the output
    # stage's header statistics of a volume restored into a SIRT run (tg_sirt_restore, then
    # tg_sirt_end runs transform + statistics on it)
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))["min_max_mean"]
    data = np.array(g["data"], np.float32)
    mean = g["mean_num"] / g["mean_den"]
    nx = data.size
    with T.Session(nx, 1, 1, np.zeros(1, np.float32), thickness=1, sirt=1) as s:
        s.upload(data.reshape(1, 1, nx))
        assert abs(s.view_sums()[0] / nx - mean) < g["tol"]
        assert s.out_shape == (1, 1, nx)
        s.sirt_restore(data.reshape(1, 1, nx), 1)  # all iterations done: output stage only
        s.sirt_end()
        vol, st = s.download()
    np.testing.assert_array_equal(vol.reshape(-1), data)  # densweight 1, outscale 1, outadd 0
    assert st["amin"] == g["min"] and st["amax"] == g["max"]
    assert abs(st["amean"] - mean) < g["tol"]
