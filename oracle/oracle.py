"""ctypes front end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module, and only as the checker or
the timed CPU baseline: nothing in the product path calls it.

The oracle restates apps/tilt/src/main.rs of imod-rs in C++ (``ref32``: f32 in
the reference's operation order; ``ref64``: the same semantics in FP64).  Its
arithmetic is parity-unpinned against the Rust binary (no Rust toolchain, the
FFT crate rustfft 6.x is not vendored); analytic known-answer tests pin it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

FILL = {"mean": 0, "zero": 1, "edge": 2}


class OrParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("out_nx", C.c_int32), ("out_nz", C.c_int32),
        ("n_angles", C.c_int32), ("angles", C.POINTER(C.c_float)),
        ("n_xtilt", C.c_int32), ("xtilt", C.POINTER(C.c_float)),
        ("n_zfac", C.c_int32), ("zfac", C.POINTER(C.c_float)),
        ("n_local", C.c_int32), ("local", C.POINTER(C.c_float)),
        ("has_local", C.c_int32),
        ("cutoff", C.c_float), ("falloff", C.c_float),
        ("no_weight", C.c_int32), ("exact_filter_size", C.c_int32), ("hamming", C.c_int32),
        ("sirt_iters", C.c_int32), ("sirt_relax", C.c_float),
        ("no_cosine_stretch", C.c_int32), ("cosine_cubic", C.c_int32),
        ("max_cosine_tilt", C.c_float), ("log_transform", C.c_int32),
        ("densweight", C.c_float), ("outscale", C.c_float), ("outadd", C.c_float),
        ("fill_mode", C.c_int32), ("fake_sirt", C.c_int32), ("gpu_compat", C.c_int32),
    ]


class OrStats(C.Structure):
    _fields_ = [("amin", C.c_float), ("amax", C.c_float), ("amean", C.c_float)]


_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with its Makefile (gcc only; no GPU needed)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB_PATH)
        f, d, i, P = C.c_float, C.c_double, C.c_int, C.c_void_p
        sigs = {
            "or_log_transform32": (None, [P, C.c_size_t]),
            "or_view_means32": (None, [P, i, i, i, P]),
            "or_weight_table32": (None, [i, f, f, i, i, P]),
            "or_weight_table64": (None, [i, d, d, i, i, P]),
            "or_rweight32": (None, [P, i, i, f, f, i, i, i]),
            "or_rweight64": (None, [P, i, i, d, d, i, i, i]),
            "or_cosine_stretch32": (None, [P, i, i, i, P, i, i, f]),
            "or_fft32": (None, [P, i, i]),
            "or_fft64": (None, [P, i, i]),
            "or_backproject32": (i, [P, P, P, P, i, i, i]),
            "or_backproject64": (i, [P, P, P, P, i, i, i]),
            "or_forward_project32": (i, [P, P, P]),
            "or_forward_project64": (i, [P, P, P]),
            "or_lowpass32": (None, [P, i, i, i]),
            "or_lowpass64": (None, [P, i, i, i]),
            "or_run32": (i, [P, P, P, P, i]),
            "or_run64": (i, [P, P, P, P, i]),
            "or_run64g": (i, [P, P, P, P, i]),
            "or_backproject64g": (i, [P, P, P, P, i, i, i]),
            "or_forward_project64g": (i, [P, P, P]),
            "or_output_stats32": (None, [P, i, i, i, f, f, f, P]),
            "or_wbp_rows32": (i, [P, P, P, i, i, i]),
            "or_wbp_rows64g": (i, [P, P, P, i, i, i]),
            "or_studio_reconstruct32": (None, [P, i, i, i, P, i, P]),
            "or_ctf_wavelength": (d, [f]),
            "or_ctf_strip_width": (i, [P, i, P, i]),
            "or_ctfphaseflip32": (i, [P, P, i, i, i, P, i, P, i, P, P]),
            "or_ctf_correct_strip32": (None, [P, P, P]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _fptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


class Params:
    """Parsed reference options (defaults of apps/tilt/src/main.rs:18-120)."""

    def __init__(self, nx, ny, nz, angles, *, width=None, thickness=0, radial=(0.35, 0.05),
                 no_weight=False, sirt=0, sirt_relax=1.0, no_cosine_stretch=False,
                 local=None, xtilt=None, zfactor=None, log=False, densweight=1.0,
                 outscale=1.0, outadd=0.0, exact_filter_size=None, fill_mode="mean",
                 cosine_interp="linear", max_cosine_tilt=80.0, hamming=False, fake_sirt=0,
                 gpu_compat=False):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.out_nx = int(width) if width else self.nx
        self.out_nz = int(thickness) if thickness and thickness > 0 else self.nx
        self.angles = np.ascontiguousarray(angles, dtype=np.float32)
        self.xtilt = None if xtilt is None else np.ascontiguousarray(xtilt, dtype=np.float32)
        self.zfactor = None if zfactor is None else np.ascontiguousarray(zfactor, dtype=np.float32)
        self.local = None if local is None else np.ascontiguousarray(local, dtype=np.float32).reshape(-1, 5)
        self.cutoff, self.falloff = float(radial[0]), float(radial[1])
        self.no_weight, self.sirt, self.sirt_relax = bool(no_weight), int(sirt), float(sirt_relax)
        self.no_cosine_stretch = bool(no_cosine_stretch)
        self.cosine_cubic = cosine_interp.lower() == "cubic"
        self.max_cosine_tilt = float(max_cosine_tilt)
        self.log = bool(log)
        self.densweight, self.outscale, self.outadd = float(densweight), float(outscale), float(outadd)
        self.exact_filter_size = int(exact_filter_size) if exact_filter_size else 0
        self.fill_mode = FILL.get(fill_mode.lower(), 0)
        self.hamming, self.fake_sirt, self.gpu_compat = bool(hamming), int(fake_sirt), bool(gpu_compat)

    def struct(self) -> OrParams:
        s = OrParams()
        s.nx, s.ny, s.nz, s.out_nx, s.out_nz = self.nx, self.ny, self.nz, self.out_nx, self.out_nz
        s.n_angles, s.angles = len(self.angles), _fptr(self.angles)
        if self.xtilt is not None:
            s.n_xtilt, s.xtilt = len(self.xtilt), _fptr(self.xtilt)
        if self.zfactor is not None:
            s.n_zfac, s.zfac = len(self.zfactor), _fptr(self.zfactor)
        if self.local is not None:
            s.n_local, s.local, s.has_local = len(self.local), _fptr(self.local), 1
        s.cutoff, s.falloff = self.cutoff, self.falloff
        s.no_weight, s.exact_filter_size, s.hamming = int(self.no_weight), self.exact_filter_size, int(self.hamming)
        s.sirt_iters, s.sirt_relax = self.sirt, self.sirt_relax
        s.no_cosine_stretch, s.cosine_cubic = int(self.no_cosine_stretch), int(self.cosine_cubic)
        s.max_cosine_tilt, s.log_transform = self.max_cosine_tilt, int(self.log)
        s.densweight, s.outscale, s.outadd = self.densweight, self.outscale, self.outadd
        s.fill_mode, s.fake_sirt, s.gpu_compat = self.fill_mode, self.fake_sirt, int(self.gpu_compat)
        s._keep = self  # arrays referenced by pointer stay alive
        return s


def run(params: Params, proj: np.ndarray, precision=32, nthreads: int = 0):
    """Whole path (main.rs:607-1093).  Returns (volume [ny][out_nz][out_nx], stats dict).

    precision: 32 (ref32), 64 (ref64: FP64 everything) or "64g" (ref64g: FP64
    data path with the reference's f32 sampling geometry)."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    assert proj.size == params.nx * params.ny * params.nz
    nthreads = nthreads or os.cpu_count() or 1
    s = params.struct()
    st = OrStats()
    shape = (params.ny, params.out_nz, params.out_nx)
    if precision == 32:
        vol = np.zeros(shape, np.float32)
        rc = lib().or_run32(C.byref(s), _ptr(proj), _ptr(vol), C.byref(st), nthreads)
    else:
        vol = np.zeros(shape, np.float64)
        fn = lib().or_run64g if precision == "64g" else lib().or_run64
        rc = fn(C.byref(s), _ptr(proj), _ptr(vol), C.byref(st), nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle run failed with code {rc}")
    return vol, {"amin": st.amin, "amax": st.amax, "amean": st.amean}


def weight_table(n, cutoff, falloff, exact_filter_size=0, hamming=False, precision=32):
    if precision == 32:
        w = np.zeros(n, np.float32)
        lib().or_weight_table32(n, cutoff, falloff, exact_filter_size or 0, int(hamming), _ptr(w))
    else:
        w = np.zeros(n, np.float64)
        lib().or_weight_table64(n, cutoff, falloff, exact_filter_size or 0, int(hamming), _ptr(w))
    return w


def rweight(rows: np.ndarray, cutoff=0.35, falloff=0.05, exact_filter_size=0, hamming=False,
            precision=32, nthreads=0):
    """apply_rweighting on a copy of rows [..., nx]."""
    nthreads = nthreads or os.cpu_count() or 1
    dt = np.float32 if precision == 32 else np.float64
    out = np.array(rows, dtype=dt, copy=True, order="C")
    nx = out.shape[-1]
    nrows = out.size // nx
    fn = lib().or_rweight32 if precision == 32 else lib().or_rweight64
    fn(_ptr(out), nx, nrows, cutoff, falloff, exact_filter_size or 0, int(hamming), nthreads)
    return out


def fft(x: np.ndarray, inverse=False, precision=32):
    dt = np.complex64 if precision == 32 else np.complex128
    a = np.array(x, dtype=dt, copy=True)
    (lib().or_fft32 if precision == 32 else lib().or_fft64)(_ptr(a), a.size, int(inverse))
    return a


def cosine_stretch(proj: np.ndarray, angles, cubic=False, max_tilt=80.0):
    a = np.array(proj, dtype=np.float32, copy=True, order="C")
    nz, ny, nx = a.shape
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    lib().or_cosine_stretch32(_ptr(a), nx, ny, nz, _ptr(ang), len(ang), int(cubic), max_tilt)
    return a


def view_means(proj: np.ndarray):
    a = np.ascontiguousarray(proj, dtype=np.float32)
    nz, ny, nx = a.shape
    m = np.zeros(nz, np.float32)
    lib().or_view_means32(_ptr(a), nx, ny, nz, _ptr(m))
    return m


def backproject(params: Params, proj: np.ndarray, means: np.ndarray, precision=32, y0=0, y1=None,
                nthreads=0):
    """WBP core on an already filtered/stretched stack (main.rs:756-828)."""
    nthreads = nthreads or os.cpu_count() or 1
    y1 = params.ny if y1 is None else y1
    dt = np.float32 if precision == 32 else np.float64
    pr = np.ascontiguousarray(proj, dtype=dt)
    mn = np.ascontiguousarray(means, dtype=dt)
    vol = np.zeros((y1 - y0, params.out_nz, params.out_nx), dt)
    s = params.struct()
    fn = {32: lib().or_backproject32, 64: lib().or_backproject64,
          "64g": lib().or_backproject64g}[precision]
    fn(C.byref(s), _ptr(pr), _ptr(mn), _ptr(vol), y0, y1, nthreads)
    return vol


def forward_project(params: Params, vol: np.ndarray, precision=32):
    dt = np.float32 if precision == 32 else np.float64
    v = np.ascontiguousarray(vol, dtype=dt)
    sino = np.zeros((params.nz, params.ny, params.nx), dt)
    s = params.struct()
    fn = {32: lib().or_forward_project32, 64: lib().or_forward_project64,
          "64g": lib().or_forward_project64g}[precision]
    fn(C.byref(s), _ptr(v), _ptr(sino))
    return sino


def lowpass(vol: np.ndarray, precision=32):
    dt = np.float32 if precision == 32 else np.float64
    v = np.array(vol, dtype=dt, copy=True, order="C")
    ny, nz, nx = v.shape
    (lib().or_lowpass32 if precision == 32 else lib().or_lowpass64)(_ptr(v), nx, nz, ny)
    return v


def output_stats(vol: np.ndarray, densweight=1.0, outscale=1.0, outadd=0.0):
    v = np.array(vol, dtype=np.float32, copy=True, order="C")
    ny, nz, nx = v.shape
    st = OrStats()
    lib().or_output_stats32(_ptr(v), nx, nz, ny, densweight, outscale, outadd, C.byref(st))
    return v, {"amin": st.amin, "amax": st.amax, "amean": st.amean}


def wbp_rows(params: Params, proj: np.ndarray, y0: int, y1: int, nthreads=0, precision=32):
    """The reference's WBP flow for slices [y0, y1) (means over whole views).

    precision 32: ref32, the timed CPU baseline; "64g": FP64 data path with the
    reference's f32 sampling geometry (error checks of the half-staging forms)."""
    nthreads = nthreads or os.cpu_count() or 1
    p = np.ascontiguousarray(proj, dtype=np.float32)
    dt = np.float32 if precision == 32 else np.float64
    vol = np.zeros((y1 - y0, params.out_nz, params.out_nx), dt)
    s = params.struct()
    fn = lib().or_wbp_rows32 if precision == 32 else lib().or_wbp_rows64g
    rc = fn(C.byref(s), _ptr(p), _ptr(vol), y0, y1, nthreads)
    if rc != 0:
        raise RuntimeError(f"oracle wbp_rows failed with code {rc}")
    return vol


def studio_reconstruct(proj: np.ndarray, angles) -> np.ndarray:
    """imod-studio's reconstruction step (apps/imod-studio/src/main.rs:725-776):
    returns [ny][nx][nx] float32."""
    p = np.ascontiguousarray(proj, dtype=np.float32)
    nz, ny, nx = p.shape
    a = np.ascontiguousarray(angles, dtype=np.float32)
    out = np.zeros((ny, nx, nx), np.float32)
    lib().or_studio_reconstruct32(_ptr(p), nx, ny, nz, _ptr(a), len(a), _ptr(out))
    return out


class CtfParams(C.Structure):
    """ctfphaseflip's options (apps/ctfphaseflip/src/main.rs:19-88 defaults)."""
    _fields_ = [("defocus", C.c_float), ("voltage", C.c_float), ("cs", C.c_float), ("pixel_a", C.c_float),
                ("strip_width", C.c_int32), ("tilt_axis_angle", C.c_float), ("max_strip_width", C.c_int32),
                ("amplitude_contrast", C.c_float), ("cuton_freq", C.c_float), ("plate_phase", C.c_float)]

    def __init__(self, **kw):
        d = dict(defocus=-3000.0, voltage=300.0, cs=2.7, pixel_a=1.0, strip_width=256, tilt_axis_angle=0.0,
                 max_strip_width=0, amplitude_contrast=0.07, cuton_freq=0.0, plate_phase=0.0)
        d.update(kw)
        super().__init__(**d)


class CtfStrip(C.Structure):
    """The shader's Params of apps/ctfphaseflip/src/ctf_correct.wgsl."""
    _fields_ = [("sw", C.c_uint32), ("sh", C.c_uint32), ("pixel_a", C.c_float), ("wavelength", C.c_float),
                ("cs_a", C.c_float), ("amp_contrast", C.c_float), ("cuton_freq", C.c_float),
                ("defocus1", C.c_float), ("defocus2", C.c_float), ("astig_angle_rad", C.c_float),
                ("has_astigmatism", C.c_uint32), ("plate_phase_rad", C.c_float), ("tilt_axis_rad", C.c_float)]


def ctf_wavelength(kv):
    return lib().or_ctf_wavelength(kv)


def ctf_strip_width(params: CtfParams, nx, view_def=None):
    vd = None if view_def is None else np.ascontiguousarray(view_def, dtype=np.float32).reshape(-1, 3)
    return lib().or_ctf_strip_width(C.byref(params), nx, _ptr(vd), 0 if vd is None else len(vd))


def ctfphaseflip(params: CtfParams, stack: np.ndarray, angles, view_def=None):
    """ctfphaseflip of a [nz][ny][nx] stack (main.rs:231-700).  Returns (out, stats)."""
    st_in = np.ascontiguousarray(stack, dtype=np.float32)
    nz, ny, nx = st_in.shape
    a = np.ascontiguousarray(angles, dtype=np.float32)
    vd = None if view_def is None else np.ascontiguousarray(view_def, dtype=np.float32).reshape(-1, 3)
    out = np.empty_like(st_in)
    st = OrStats()
    lib().or_ctfphaseflip32(C.byref(params), _ptr(st_in), nx, ny, nz, _ptr(a), len(a), _ptr(vd),
                            0 if vd is None else len(vd), _ptr(out), C.byref(st))
    return out, {"amin": st.amin, "amax": st.amax, "amean": st.amean}


def ctf_correct_strip(re, im, strip: CtfStrip):
    """ctf_correct.wgsl in f32 on one strip's re/im (copies returned)."""
    r = np.array(re, dtype=np.float32, copy=True, order="C")
    i = np.array(im, dtype=np.float32, copy=True, order="C")
    lib().or_ctf_correct_strip32(_ptr(r), _ptr(i), C.byref(strip))
    return r, i
