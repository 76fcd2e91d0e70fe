"""Failure detection on the device without a device fault.

The pipelined back-projector's waits (its producer warp's copies completing on
mbarriers, the consumers releasing ring slots) are bounded: after the limit the
CTA records the timeout in the session's error word, waits (bounded) for its own
copies in flight and returns; tg_synchronize reports TG_ERR_TIMEOUT.  The test
hook makes the producer leave out one pipeline stage (no copy is issued, so its
barrier phase never completes) with a 5 ms limit: the timeout path runs, nothing
faults, and the same session then reconstructs normally again.
"""
import time

import numpy as np
import pytest

import oracle as O
import tiltgpu as T
from tgutil import angles, rel_l2, smooth_stack

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_bounded_wait_times_out_and_session_recovers(storage):
    nz, ny, nx = 31, 16, 128
    proj = smooth_stack(nz, ny, nx, seed=91)
    ang = angles(-60, 60, 4)
    kw = dict(thickness=48, radial=(0.35, 0.035), storage=storage)
    with T.Session(nx, ny, nz, ang, **kw) as s:
        assert s.kernel_info()["fast"]
        s.upload(proj)
        s.reconstruct()  # tunes the tile shape with the normal limit
        good, _ = s.download()
        s.inject_wait_fault(skip_stage=1, wait_limit_us=5000)
        t0 = time.perf_counter()
        with pytest.raises(T.TiltGpuError) as e:
            s.reconstruct()
        assert e.value.code == -4 and "timed out" in str(e.value)
        assert time.perf_counter() - t0 < 30.0
        s.inject_wait_fault(-1, 0)
        s.reconstruct()
        again, _ = s.download()
    np.testing.assert_array_equal(again, good)
    ref, _ = O.run(O.Params(nx, ny, nz, ang, thickness=48, radial=(0.35, 0.035)), proj,
                   32 if storage == "fp32" else "64g")
    assert rel_l2(good, ref) <= (1e-5 if storage == "fp32" else 2e-3)


def test_wait_fault_hook_needs_the_pipelined_kernel():
    nz, ny, nx = 9, 4, 32
    ang = angles(-40, 40, 10)
    with T.Session(nx, ny, nz, ang, thickness=16, xtilt=np.linspace(-2, 2, nz).astype(np.float32)) as s:
        with pytest.raises(T.TiltGpuError) as e:  # per-view x-tilts: another back-projector
            s.inject_wait_fault(1, 5000)
        assert e.value.code == -6
