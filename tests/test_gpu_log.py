"""The --log transform on the device (apps/tilt/src/main.rs:606-612:
v.max(0.001).log10() in f32) gives the correctly rounded f32 logarithm on
every sample, over the whole f32 range the data can take: the table-driven
evaluation decides most samples and hands those near a rounding boundary to
the double-precision library log10.

One view at 0 degrees, no weighting, no stretch, one slice thick: every voxel
but the last column of a row is its sample (the back-projector's fraction is 0
and 1/N is 1), so the volume shows the logged samples themselves.  The
expected values are the float32 rounding of log10 in x87 extended precision;
the few samples whose extended value lies within 2^-50 of a midpoint between
floats (where even an FP64 log10 may round either way) are left out."""
import numpy as np
import pytest

import tiltgpu as T

pytestmark = pytest.mark.gpu


def samples(rng, n):
    parts = [
        (10.0 ** rng.uniform(-4.5, 7.5, n)).astype(np.float32),   # six-plus decades of counts
        np.arange(0, 65536, dtype=np.float32),                     # integer counts
        (1.0 + np.arange(-4000, 4000) * 2.0 ** -24).astype(np.float32),  # around 1 (log near 0)
        np.array([0.0, -1.0, -1e30, 1e-30, 0.000999, 0.001, 0.0010001, 3.0e38], np.float32),
    ]
    # the table's bucket edges and centres in many binades, with their neighbours
    j = np.arange(257, dtype=np.int64)
    pats = []
    for e in range(-10, 40):
        centre = 0x3F400000 + j * (1 << 15) + (e << 23)
        edge = centre + (1 << 14)
        for d in (-2, -1, 0, 1, 2):
            pats.append(centre + d)
            pats.append(edge + d)
    pats = np.concatenate(pats)
    pats = pats[(pats > 0) & (pats < 0x7F800000)].astype(np.uint32).view(np.float32)
    parts.append(pats)
    return np.concatenate(parts)


def test_log_transform_correctly_rounded():
    if np.finfo(np.longdouble).nmant < 63:
        pytest.skip("needs x87 extended precision for the expected values")
    rng = np.random.default_rng(12)
    nx = 2048
    x = samples(rng, 6_000_000)
    ny = -(-x.size // nx)
    x = np.concatenate([x, np.full(ny * nx - x.size, 7.0, np.float32)])
    rng.shuffle(x)
    proj = x.reshape(1, ny, nx)
    xc = np.maximum(x, np.float32(0.001)).astype(np.longdouble)
    L = np.log10(xc)
    want = L.astype(np.float32)
    # midpoints to the neighbours of the rounded value; within 2^-50 is ambiguous
    up = np.nextafter(want, np.float32(np.inf)).astype(np.longdouble)
    dn = np.nextafter(want, np.float32(-np.inf)).astype(np.longdouble)
    w = want.astype(np.longdouble)
    tol = np.abs(L) * np.longdouble(2.0 ** -50)
    ambiguous = (np.abs(L - (w + up) / 2) < tol) | (np.abs(L - (w + dn) / 2) < tol)
    opts = dict(thickness=1, no_weight=True, no_cosine_stretch=True, fill_mode="zero")
    vol, _ = T.reconstruct(proj, np.zeros(1, np.float32), log=True, **opts)
    got = vol[:, 0, :].reshape(-1)
    keep = np.ones(ny * nx, bool)
    keep[nx - 1::nx] = False          # the last column of a row is the fill
    keep &= ~ambiguous
    assert keep.sum() > 0.999 * (ny * (nx - 1))
    bad = np.flatnonzero(keep & (got.view(np.uint32) != want.view(np.uint32)))
    assert bad.size == 0, (bad.size, x[bad[:5]], got[bad[:5]], want[bad[:5]])
    # the same path without --log on the expected values gives the same volume
    vol2, _ = T.reconstruct(want.reshape(1, ny, nx), np.zeros(1, np.float32), **opts)
    np.testing.assert_array_equal(vol2.reshape(-1)[keep], got[keep])
