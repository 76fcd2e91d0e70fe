"""Multi-process plumbing for the tilt path (one process per GPU).

Without x-tilt or local alignment every output slice iy reads only projection
row iy of each view (apps/tilt/src/main.rs:1047-1065), so a series splits into
independent Y slabs with no data-path exchange; only the header statistics
need combining, which is done here in the reference's slice order
(apps/tilt/src/main.rs:1077-1093).  Independent series per rank need nothing
but the timing reduction (max over ranks) and the update count (sum).
"""
from __future__ import annotations

import numpy as np


def slab_bounds(ny: int, world: int, rank: int, align: int = 8):
    """Contiguous [y0, y1) of rank, slab edges on multiples of `align` slices."""
    blocks = (ny + align - 1) // align
    b0 = blocks * rank // world
    b1 = blocks * (rank + 1) // world
    return min(ny, b0 * align), min(ny, b1 * align)


def combine_slice_stats(slice_stats, count: int):
    """Header (amin, amax, amean) from per-slice (min, max, f32 mean) in Y order."""
    gmin, gmax, gsum = np.float32(3.4028235e38), np.float32(-3.4028235e38), 0.0
    for mn, mx, mean in slice_stats:
        if np.float32(mn) < gmin:
            gmin = np.float32(mn)
        if np.float32(mx) > gmax:
            gmax = np.float32(mx)
        gsum += float(np.float32(mean)) * count
    n = len(slice_stats)
    return float(gmin), float(gmax), float(np.float32(gsum / (count * n))) if n else 0.0


def slice_stats(vol: np.ndarray):
    """Per-slice (min, max, f32 mean with an f64 sum) of a [y][z][x] f32 block."""
    out = []
    for s in vol:
        out.append((float(s.min()), float(s.max()), float(np.float32(s.astype(np.float64).sum() / s.size))))
    return out


def gather_stats(local, y0: int, group=None):
    """All ranks' (y0, per-slice stats) gathered and folded in Y order."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, (y0, local), group=group)
    parts.sort(key=lambda p: p[0])
    merged = [s for _, st in parts for s in st]
    return merged


def whole_series_means(view_sums, nx: int, ny_total: int):
    """Mean fill values of whole views from the per-view f64 sums of all slabs
    (apps/tilt/src/main.rs:616-623: the f64 mean rounded to f32)."""
    return (np.asarray(view_sums, np.float64) / float(nx * ny_total)).astype(np.float32)


def all_reduce_sums(x, group=None):
    """Element-wise sum of a float64 vector over the ranks."""
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.ascontiguousarray(x, np.float64)).clone()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.numpy()


def reconstruct_slab(proj_slab, angles, nx: int, ny_total: int, sum_views=all_reduce_sums, **opts):
    """One rank's Y slab of a series through the CUDA path: upload the slab's rows,
    add the per-view sums over the ranks (sum_views), pin the whole series' mean fill
    values, reconstruct.  Returns the slab's volume and its per-slice statistics.
    Not for x-tilt, local alignment or fake SIRT (their rows or slices reach across
    slab edges)."""
    import tiltgpu as T

    nz, ny, _ = proj_slab.shape
    with T.Session(nx, ny, nz, angles, **opts) as s:
        s.upload(proj_slab)
        s.set_view_means(whole_series_means(sum_views(s.view_sums()), nx, ny_total))
        s.reconstruct()
        vol, _ = s.download()
    return vol, slice_stats(vol)


def reduce_max(x: float, group=None) -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def reduce_sum(x: float, group=None) -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
