"""Serving: jobs submitted while others run are admitted by a memory budget,
batched per round, and each result is the same as the series reconstructed alone.
Failures are injected on the host (allocation, admission); no device fault."""
import threading

import numpy as np
import pytest

import tiltgpu as T
from tgutil import smooth_stack

pytestmark = pytest.mark.gpu

JOBS = [
    dict(nx=96, ny=24, nz=31, thickness=40, storage="fp16"),
    dict(nx=64, ny=17, nz=21, thickness=33, storage="fp32"),
    dict(nx=128, ny=16, nz=41, thickness=50, storage="fp16", sirt=3),
    dict(nx=80, ny=12, nz=19, thickness=28, storage="fp32", zfactor=True),
    dict(nx=64, ny=10, nz=15, thickness=20, storage="fp32", xtilt=True, sirt=2),
    dict(nx=100, ny=9, nz=25, thickness=30, storage="bf16", width=90),
    dict(nx=48, ny=8, nz=11, thickness=16, storage="fp16", fake_sirt=1),
    dict(nx=72, ny=20, nz=27, thickness=36, storage="fp32", sirt=2),
]


def spec(job, seed):
    nx, ny, nz = job["nx"], job["ny"], job["nz"]
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    kw = dict(thickness=job["thickness"], storage=job["storage"], sirt=job.get("sirt", 0),
              fake_sirt=job.get("fake_sirt", 0), width=job.get("width"), radial=(0.35, 0.035))
    if job.get("zfactor"):
        kw["zfactor"] = np.linspace(0.9, 1.1, nz).astype(np.float32)
    if job.get("xtilt"):
        kw["xtilt"] = np.full(nz, 1.5, np.float32)
    return smooth_stack(nz, ny, nx, seed=seed), ang, kw


def out_shape(job):
    return (job["ny"], job["thickness"], job.get("width") or job["nx"])


@pytest.fixture(scope="module")
def alone():
    res = []
    for i, job in enumerate(JOBS):
        proj, ang, kw = spec(job, 100 + i)
        res.append(T.reconstruct(proj, ang, **kw))
    return res


def check_same(vol, st, ref):
    va, sa = ref
    np.testing.assert_array_equal(vol, va)
    assert st["amin"] == sa["amin"] and st["amax"] == sa["amax"]
    assert abs(st["amean"] - sa["amean"]) <= 1e-6 * max(1e-6, abs(sa["amean"]))


def test_mix_equals_alone(alone):
    with T.Server(budget_bytes=0, max_active=16) as sv:
        ids, outs = [], []
        for rep in range(2):  # the second wave arrives while the first still runs
            for i, job in enumerate(JOBS):
                proj, ang, kw = spec(job, 100 + i)
                out = np.empty(out_shape(job), np.float32)
                ids.append(sv.submit(proj, ang, out=out, tag=i, **kw))
                outs.append(out)
        for jid, out in zip(ids, outs):
            r = sv.wait(jid, 60000)
            assert r is not None and r["state"] == "done", r
            check_same(out, r["stats"], alone[r["tag"]])
            assert r["done_ms"] >= r["admit_ms"] >= r["submit_ms"] >= 0
            sv.release(jid)
        info = sv.info()
        assert info["completed"] == len(ids) and info["failed"] == 0
        assert info["bytes_in_use"] == 0
        assert info["rounds"] >= 4  # SIRT jobs take one round per iteration


def test_budget_admission_and_threads(alone):
    # a budget that holds about two of the jobs at a time: the rest queue
    sizes = []
    for i, job in enumerate(JOBS):
        proj, ang, kw = spec(job, 100 + i)
        with T.Session(job["nx"], job["ny"], job["nz"], ang, **{k: v for k, v in kw.items()}) as s:
            sizes.append(s.device_bytes())
    budget = int(2.2 * max(sizes))
    with T.Server(budget_bytes=budget, max_active=8) as sv:
        results = {}
        lock = threading.Lock()

        def client(idx):
            for i in idx:
                proj, ang, kw = spec(JOBS[i], 100 + i)
                out = np.empty(out_shape(JOBS[i]), np.float32)
                jid = sv.submit(proj, ang, out=out, tag=i, **kw)
                r = sv.wait(jid, 60000)
                with lock:
                    results[i] = (out, r)

        ths = [threading.Thread(target=client, args=(list(range(k, len(JOBS), 3)),)) for k in range(3)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        assert sorted(results) == list(range(len(JOBS)))
        for i, (out, r) in results.items():
            assert r["state"] == "done", r
            check_same(out, r["stats"], alone[i])
        info = sv.info()
        assert 0 < info["bytes_peak"] <= budget
        # a job that can never fit is refused at submission
        proj, ang, kw = spec(JOBS[0], 1)
        tiny = T.Server(budget_bytes=1 << 20)
        with pytest.raises(T.TiltGpuError) as e:
            tiny.submit(proj, ang, **kw)
        assert e.value.code == -5
        tiny.close()


def test_injected_failures_do_not_disturb_others(alone):
    with T.Server(max_active=4) as sv:
        sv.inject(T.FAULT_ALLOC, 1)
        proj, ang, kw = spec(JOBS[1], 101)
        bad = sv.submit(proj, ang, out=np.empty(out_shape(JOBS[1]), np.float32), **kw)
        r = sv.wait(bad, 60000)
        assert r["state"] == "failed" and r["status"] == -2
        sv.inject(T.FAULT_ADMIT, 1)
        refused = sv.submit(proj, ang, **kw)
        r = sv.wait(refused, 60000)
        assert r["state"] == "failed" and r["status"] == -5
        ok = []
        for i in (0, 2, 4):
            proj, ang, kw = spec(JOBS[i], 100 + i)
            out = np.empty(out_shape(JOBS[i]), np.float32)
            ok.append((i, out, sv.submit(proj, ang, out=out, **kw)))
        for i, out, jid in ok:
            r = sv.wait(jid, 60000)
            assert r["state"] == "done"
            check_same(out, r["stats"], alone[i])
        info = sv.info()
        assert info["failed"] == 2 and info["completed"] == 3


def test_destroy_cancels_queued():
    sv = T.Server(budget_bytes=0, max_active=1)
    proj, ang, kw = spec(JOBS[2], 7)  # SIRT: keeps the single slot busy for a few rounds
    ids = [sv.submit(proj, ang, **kw) for _ in range(6)]
    sv.close()  # running job finishes, queued ones are dropped; no hang
