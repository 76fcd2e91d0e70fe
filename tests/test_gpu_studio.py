"""imod-studio's reconstruction step through tg_studio_reconstruct.

step_reconstruction (apps/imod-studio/src/main.rs:725-776) is an unweighted,
unstretched, zero-fill back-projection of <base>.ali along <base>.tlt into
<base>_full.rec.  The CUDA path (files in, files out, through the C ABI) must
give the oracle's direct restatement of those lines bit for bit, with the
step's header (MrcHeader::new(nx, nx, ny, Float), its label, statistics 0).
"""
import numpy as np
import pytest

import oracle as O
import tiltgpu as T
from tgutil import random_stack

pytestmark = pytest.mark.gpu


def write_dataset(tmp_path, proj, ang):
    nz, ny, nx = proj.shape
    ali, tlt, rec = tmp_path / "ds.ali", tmp_path / "ds.tlt", tmp_path / "ds_full.rec"
    T.mrc_write_f32(ali, T.mrc_header_new(nx, ny, nz, "Float"), proj)
    T.write_tilt_file(tlt, ang)
    return ali, tlt, rec


@pytest.mark.parametrize("shape", [(15, 6, 48), (21, 4, 100)])
def test_studio_step_bit_exact(tmp_path, shape):
    nz, ny, nx = shape
    proj = random_stack(nz, ny, nx, seed=nx, offset=-0.3)
    ang = np.round(np.linspace(-58, 58, nz), 2).astype(np.float32)  # the .tlt holds 2 decimals
    ali, tlt, rec = write_dataset(tmp_path, proj, ang)
    T.studio_reconstruct(ali, tlt, rec)
    info, data = T.mrc_read(rec)
    assert (info.nx, info.ny, info.nz, info.mode) == (nx, nx, ny, 2)
    assert (info.amin, info.amax, info.amean) == (0.0, 0.0, 0.0)
    assert b"imod-studio: reconstruction" in bytes(info.header[224:304])
    want = O.studio_reconstruct(proj, T.read_tilt_file(tlt))
    np.testing.assert_array_equal(data.reshape(ny, nx, nx), want)


def test_studio_step_missing_files(tmp_path):
    proj = random_stack(5, 2, 16, seed=1)
    ali, tlt, rec = write_dataset(tmp_path, proj, np.zeros(5, np.float32))
    with pytest.raises(T.TiltGpuError) as e:
        T.studio_reconstruct(tmp_path / "nope.ali", tlt, rec)
    assert e.value.code == -1 and "not found" in str(e.value)
    with pytest.raises(T.TiltGpuError) as e:
        T.studio_reconstruct(ali, tmp_path / "nope.tlt", rec)
    assert "not found" in str(e.value)
