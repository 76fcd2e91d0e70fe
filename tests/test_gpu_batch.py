"""Batched reconstruction: one persistent back-projection launch per round over
many uneven series gives every series exactly its stand-alone volume."""
import numpy as np
import pytest

import tiltgpu as T
from tgutil import smooth_stack

pytestmark = pytest.mark.gpu

JOBS = [
    dict(nx=96, ny=24, nz=31, thickness=40, storage="fp16"),
    dict(nx=64, ny=17, nz=21, thickness=33, storage="fp32"),
    dict(nx=128, ny=16, nz=41, thickness=50, storage="fp16", sirt=2),
    dict(nx=80, ny=12, nz=19, thickness=28, storage="fp32", zfactor=True),
    dict(nx=64, ny=10, nz=15, thickness=20, storage="fp32", xtilt=True),
    dict(nx=100, ny=9, nz=25, thickness=30, storage="bf16", width=90),
    dict(nx=48, ny=8, nz=11, thickness=16, storage="fp16", fake_sirt=1),
]


def make(job, seed):
    nx, ny, nz = job["nx"], job["ny"], job["nz"]
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    kw = dict(thickness=job["thickness"], storage=job["storage"], sirt=job.get("sirt", 0),
              fake_sirt=job.get("fake_sirt", 0), width=job.get("width"))
    if job.get("zfactor"):
        kw["zfactor"] = np.linspace(0.9, 1.1, nz).astype(np.float32)
    if job.get("xtilt"):
        kw["xtilt"] = np.full(nz, 1.5, np.float32)
    s = T.Session(nx, ny, nz, ang, **kw)
    s.upload(smooth_stack(nz, ny, nx, seed=seed))
    return s


def test_batch_equals_stand_alone():
    alone = []
    for i, job in enumerate(JOBS):
        s = make(job, i)
        s.reconstruct()
        alone.append(s.download())
        s.close()
    sessions = [make(job, i) for i, job in enumerate(JOBS)]
    b = T.Batch()
    for s in sessions:
        b.add(s)
    for rep in range(2):  # twice: resident projections, repeatable results
        b.reconstruct()
        for (va, sa), s in zip(alone, sessions):
            vb, sb = s.download()
            np.testing.assert_array_equal(vb, va)
            assert sb["amin"] == sa["amin"] and sb["amax"] == sa["amax"]
            assert abs(sb["amean"] - sa["amean"]) <= 1e-6 * max(1e-6, abs(sa["amean"]))
    info = b.last_run()
    assert info["passes"] == 3 and info["updates"] > 0
    b.close()
    for s in sessions:
        s.close()


SIRT_JOBS = [  # every reprojection form and filter width group, uneven iteration counts
    dict(nx=256, ny=12, nz=31, thickness=40, storage="fp16", sirt=3),
    dict(nx=256, ny=9, nz=25, thickness=36, storage="fp16", sirt=2),
    dict(nx=384, ny=10, nz=21, thickness=30, storage="fp16", sirt=3, xtilt=True),
    dict(nx=256, ny=11, nz=27, thickness=44, storage="fp32", sirt=3),
    dict(nx=384, ny=8, nz=19, thickness=28, storage="fp32", sirt=2, xtilt=True),
    dict(nx=256, ny=10, nz=23, thickness=32, storage="bf16", sirt=3),
    dict(nx=100, ny=8, nz=17, thickness=24, storage="fp32", sirt=2),   # generic filter width
    dict(nx=96, ny=9, nz=15, thickness=20, storage="fp16", sirt=1),
]


@pytest.mark.parametrize("grouped_fp", [False, True])
def test_batched_sirt_rounds_grouped_and_graphed(grouped_fp, monkeypatch):
    # SIRT rounds run as grouped reprojection / filter / back-projection launches,
    # replayed from a CUDA graph while the members stay the same; every series must
    # still come out bit-identical to its stand-alone reconstruction
    if grouped_fp:  # reprojection of same-form series in one launch per phase
        monkeypatch.setenv("TG_ROUND_FP_BATCH", "1")
    alone = []
    for i, job in enumerate(SIRT_JOBS):
        s = _make_relaxed(job, 100 + i)
        s.reconstruct()
        alone.append(s.download())
        s.close()
    sessions = [_make_relaxed(job, 100 + i) for i, job in enumerate(SIRT_JOBS)]
    b = T.Batch()
    for s in sessions:
        b.add(s)
    for rep in range(2):
        b.reconstruct()
        for (va, sa), s in zip(alone, sessions):
            vb, sb = s.download()
            np.testing.assert_array_equal(vb, va)
            assert sb["amin"] == sa["amin"] and sb["amax"] == sa["amax"]
    info = b.plan_info()
    assert info["graph_rounds"] == 3          # rounds 1..3, one plan per member list
    assert (info["fp_groups"] >= 2) == grouped_fp and info["filter_groups"] >= 1
    b.close()
    for s in sessions:
        s.close()


def _make_relaxed(job, seed):
    nx, ny, nz = job["nx"], job["ny"], job["nz"]
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    kw = dict(thickness=job["thickness"], storage=job["storage"], sirt=job.get("sirt", 0), sirt_relax=0.5)
    if job.get("xtilt"):
        kw["xtilt"] = np.full(nz, 1.5, np.float32)
    s = T.Session(nx, ny, nz, ang, **kw)
    s.upload(smooth_stack(nz, ny, nx, seed=seed))
    return s
