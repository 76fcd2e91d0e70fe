"""Y slabs of one series through the CUDA path (what one rank per GPU runs)
give the single-process volume and header statistics.  Two ranks are emulated
one after the other on one GPU: their per-view sums are added on the host, as
the all-reduce of shard.reconstruct_slab adds them across ranks.  (Fake SIRT's
3-tap filter across slices couples neighbouring slabs and is not sharded.)"""
import numpy as np
import pytest

import shard
import tiltgpu as T
from tgutil import angles, rel_l2, smooth_stack

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world,kw", [(2, dict(log=True)), (3, dict(storage="fp16")),
                                      (2, dict(sirt=2, sirt_relax=0.5, zfactor=None))])
def test_slabs_reproduce_the_whole_series(world, kw):
    nz, ny, nx = 17, 40, 96
    proj = (smooth_stack(nz, ny, nx, seed=world) * 300.0 + 20000.0).astype(np.float32)
    ang = angles(-56, 56, 7)
    opts = dict(thickness=36, radial=(0.35, 0.035), **{k: v for k, v in kw.items() if v is not None})
    whole, wst = T.reconstruct(proj, ang, **opts)
    # pass 1: every rank's per-view sums (the all-reduce), pass 2: the slabs with pinned means
    bounds = [shard.slab_bounds(ny, world, r) for r in range(world)]
    sums = np.zeros(nz, np.float64)
    for y0, y1 in bounds:
        with T.Session(nx, y1 - y0, nz, ang, **opts) as s:
            s.upload(proj[:, y0:y1])
            sums += s.view_sums()
    vols, stats = [], []
    for y0, y1 in bounds:
        v, st = shard.reconstruct_slab(np.ascontiguousarray(proj[:, y0:y1]), ang, nx, ny,
                                       sum_views=lambda _local: sums, **opts)
        vols.append(v)
        stats += st
    got = np.concatenate(vols)
    assert rel_l2(got, whole) <= 1e-6, rel_l2(got, whole)
    amin, amax, amean = shard.combine_slice_stats(stats, nx * 36)
    assert amin == pytest.approx(wst["amin"], rel=1e-6) and amax == pytest.approx(wst["amax"], rel=1e-6)
    assert amean == pytest.approx(wst["amean"], rel=1e-5, abs=1e-7)
