"""The allocation-free R-weighting entry point against the allocating one.

tg_apply_rweighting_device_noalloc exists for callers that cannot call
cudaMalloc (hosts that own all device memory through their own pool, services
that must not trigger cudaMalloc's device-wide synchronisation).  It keeps its
tables in one static device array shared by all calls, so this test makes two
calls in a row with different sizes and options and checks each against
tg_apply_rweighting, which allocates a session.  Collected last on purpose
(file name), and written to pass alone in a fresh process or after the others.
"""
import numpy as np
import pytest

import tiltgpu as T
from tgutil import rel_l2, smooth_stack

pytestmark = pytest.mark.gpu

TOL = 1e-6  # same arithmetic on the same device; observed results are identical


def _noalloc(proj, **kw):
    import torch

    d = torch.from_numpy(np.ascontiguousarray(proj, dtype=np.float32)).cuda()
    nz, ny, nx = proj.shape
    stream = torch.cuda.current_stream()
    T.apply_rweighting_device_noalloc(d.data_ptr(), nx, ny, nz, stream=stream.cuda_stream, **kw)
    torch.cuda.synchronize()
    return d.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    a = smooth_stack(5, 7, 512, seed=1)  # radix-2 rows, odd row count
    b = smooth_stack(3, 4, 500, seed=2)  # radix-2/5 rows, Hamming window, explicit table size
    want_a = T.apply_rweighting(a, 0.35, 0.05)
    want_b = T.apply_rweighting(b, 0.3, 0.04, exact_filter_size=200, use_hamming=True)
    got_a = _noalloc(a, cutoff=0.35, falloff=0.05)
    got_b = _noalloc(b, cutoff=0.3, falloff=0.04, exact_filter_size=200, use_hamming=True)
    assert rel_l2(got_a, want_a) <= TOL
    assert rel_l2(got_b, want_b) <= TOL
    # the tables of the previous call are left in the shared array; a repeat must rewrite them
    got_a2 = _noalloc(a, cutoff=0.35, falloff=0.05)
    assert rel_l2(got_a2, want_a) <= TOL


def test_noalloc_rows_without_a_radix_plan():
    # 509 samples (prime): both entry points filter by circulant convolution with the
    # inverse transform of the weights, kept in the static array after the weights
    c = smooth_stack(2, 3, 509, seed=3)
    want_c = T.apply_rweighting(c, 0.35, 0.05)
    got_c = _noalloc(c, cutoff=0.35, falloff=0.05)
    assert rel_l2(got_c, want_c) <= TOL
    a = smooth_stack(5, 7, 512, seed=1)  # back to a radix plan: the convolution table is unused
    assert rel_l2(_noalloc(a, cutoff=0.35, falloff=0.05), T.apply_rweighting(a, 0.35, 0.05)) <= TOL


def test_noalloc_rejects_rows_beyond_the_static_limit():
    import torch

    d = torch.zeros(2 * 2 * 8193, dtype=torch.float32, device="cuda")
    with pytest.raises(T.TiltGpuError) as e:  # rejected on the host before any device work
        T.apply_rweighting_device_noalloc(d.data_ptr(), 8193, 2, 2)
    assert e.value.code == -1 and "8192" in str(e.value)
