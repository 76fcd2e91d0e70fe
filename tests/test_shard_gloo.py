"""Two gloo ranks on the CPU: Y-slab sharding of one series reproduces the
single-process volume and header statistics; timing/updates reductions."""
import os
import socket

import numpy as np
import pytest

import shard

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, proj, out_dir):
    import datetime

    import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    nz, ny, nx = proj.shape
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    p = O.Params(nx, ny, nz, ang, thickness=12)
    y0, y1 = shard.slab_bounds(ny, world, rank)
    vol = O.wbp_rows(p, proj, y0, y1, nthreads=2)
    out, _ = O.output_stats(vol)
    merged = shard.gather_stats(shard.slice_stats(out), y0)
    st = shard.combine_slice_stats(merged, out.shape[1] * out.shape[2])
    t = shard.reduce_max(float(rank + 1))
    u = shard.reduce_sum(1000.0 * (rank + 1))
    np.save(os.path.join(out_dir, f"vol{rank}.npy"), out)
    np.save(os.path.join(out_dir, f"st{rank}.npy"), np.array(list(st) + [t, u, y0, y1]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_slabs_match_single_process(tmp_path):
    import oracle as O
    rng = np.random.default_rng(0)
    proj = (rng.random((9, 20, 32)) + 1).astype(np.float32)
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, proj, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    nz, ny, nx = proj.shape
    ang = np.linspace(-60, 60, nz).astype(np.float32)
    ref, rst = O.run(O.Params(nx, ny, nz, ang, thickness=12), proj, 32, nthreads=2)
    vols = [np.load(tmp_path / f"vol{r}.npy") for r in range(2)]
    np.testing.assert_array_equal(np.concatenate(vols), ref)
    for r in range(2):
        st = np.load(tmp_path / f"st{r}.npy")
        assert st[0] == np.float32(rst["amin"]) and st[1] == np.float32(rst["amax"])
        assert abs(st[2] - rst["amean"]) <= 1e-7 * max(1.0, abs(rst["amean"]))
        assert st[3] == 2.0 and st[4] == 3000.0
    assert np.load(tmp_path / "st0.npy")[6] == 8  # slab edge on a multiple of 8 slices


def test_slab_bounds_cover():
    for ny in (1, 7, 8, 100, 2048):
        for world in (1, 2, 3, 8):
            b = [shard.slab_bounds(ny, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == ny
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
