"""Shared helpers for the tests (comparison metrics, seeded inputs)."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if not (np.iscomplexobj(a) or np.iscomplexobj(b)):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


def angles(lo=-60.0, hi=60.0, step=2.0):
    n = int(round((hi - lo) / step)) + 1
    return (lo + step * np.arange(n)).astype(np.float32)


def random_stack(nz, ny, nx, seed=0, offset=1.0):
    rng = np.random.default_rng(seed)
    return (rng.random((nz, ny, nx)) + offset).astype(np.float32)


def smooth_stack(nz, ny, nx, seed=0):
    """Random stack with structure at several scales (closer to real projections)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((nz, ny, nx)).astype(np.float64)
    k = np.fft.rfftfreq(nx)
    spec = np.fft.rfft(x, axis=-1) / (1.0 + (k / 0.05) ** 2)
    y = np.fft.irfft(spec, n=nx, axis=-1)
    return (y / y.std() + 3.0).astype(np.float32)
