"""Python binding of libtiltgpu.so (the C ABI declared in include/tiltgpu.h).

Mirrors the reference's `tilt` options (apps/tilt/src/main.rs:18-120) and its
GPU seam (GpuSession::new / reconstruct_row, apps/tilt/src/gpu.rs:43-269).
There is no CPU fallback: if the shared library is missing or no sm_100 GPU is
present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("TILTGPU_LIB") or os.path.join(_HERE, "lib", "libtiltgpu.so")
CLI_PATH = os.path.join(_HERE, "bin", "tilt")
CTF_CLI_PATH = os.path.join(_HERE, "bin", "ctfphaseflip")

TG_OK = 0
STATUS = {0: "ok", -1: "invalid argument", -2: "out of device memory", -3: "CUDA error",
          -4: "device wait timed out", -5: "over memory budget", -6: "unsupported",
          -7: "no sm_100 CUDA device", -8: "input on which the reference panics",
          -9: "not ready", -10: "not found", -11: "cancelled", -12: "value beyond the FP16 staging range"}
FILL = {"mean": 0, "zero": 1, "edge": 2}
STORAGE = {"fp32": 0, "fp16": 1, "bf16": 2}

_f, _i32, _P = C.c_float, C.c_int32, C.c_void_p
_fp = C.POINTER(C.c_float)


class Geometry(C.Structure):
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("out_nx", _i32), ("out_nz", _i32),
                ("n_angles", _i32), ("angles", _fp), ("n_xtilt", _i32), ("xtilt", _fp),
                ("n_zfactor", _i32), ("zfactor", _fp), ("n_local", _i32), ("local", _fp),
                ("has_local", _i32)]


class Options(C.Structure):
    _fields_ = [("radial_cutoff", _f), ("radial_falloff", _f), ("hamming", _i32),
                ("exact_filter_size", _i32), ("no_weight", _i32), ("fill_mode", _i32),
                ("no_cosine_stretch", _i32), ("cosine_cubic", _i32), ("max_cosine_tilt", _f),
                ("log_transform", _i32), ("sirt_iters", _i32), ("sirt_relax", _f),
                ("fake_sirt", _i32), ("densweight", _f), ("outscale", _f), ("outadd", _f),
                ("gpu_compat", _i32), ("storage", _i32), ("device", _i32), ("use_graphs", _i32),
                ("exact_xtilt", _i32)]


class Stats(C.Structure):
    _fields_ = [("amin", _f), ("amax", _f), ("amean", _f)]


class RunInfo(C.Structure):
    _fields_ = [("updates", C.c_double), ("ms_total", C.c_double), ("ms_filter", C.c_double),
                ("ms_backproject", C.c_double), ("ms_reproject", C.c_double), ("passes", _i32),
                ("kernel_launches", _i32)]


class PhantomSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("nx", _i32), ("ny", _i32), ("nz", _i32),
                ("vol_nx", _i32), ("vol_nz", _i32), ("n_ell", _i32), ("rmin", _f), ("rmax", _f),
                ("dmin", _f), ("dmax", _f), ("n_beads", _i32), ("bead_r", _f), ("bead_d", _f),
                ("noise_kind", _i32), ("noise", _f), ("xtilt_deg", _f)]


class CtfOptions(C.Structure):
    _fields_ = [("defocus", _f), ("voltage", _f), ("cs", _f), ("pixel_size", _f), ("strip_width", _i32),
                ("tilt_axis_angle", _f), ("max_strip_width", _i32), ("amplitude_contrast", _f),
                ("cuton_freq", _f), ("plate_phase", _f), ("device", _i32)]


class CtfStripParams(C.Structure):
    _fields_ = [("sw", C.c_uint32), ("sh", C.c_uint32), ("pixel_a", _f), ("wavelength", _f), ("cs_a", _f),
                ("amp_contrast", _f), ("cuton_freq", _f), ("defocus1", _f), ("defocus2", _f),
                ("astig_angle_rad", _f), ("has_astigmatism", C.c_uint32), ("plate_phase_rad", _f),
                ("tilt_axis_rad", _f)]


class MrcInfo(C.Structure):
    _fields_ = [("nx", _i32), ("ny", _i32), ("nz", _i32), ("mode", _i32), ("next", _i32),
                ("swapped", _i32), ("xlen", _f), ("ylen", _f), ("zlen", _f), ("amin", _f),
                ("amax", _f), ("amean", _f), ("nlabl", _i32), ("imod", _i32),
                ("header", C.c_uint8 * 1024)]


class Job(C.Structure):
    _fields_ = [("geometry", Geometry), ("options", Options), ("projections", _P),
                ("n_projections", C.c_size_t), ("volume_out", _P), ("tag", C.c_uint64)]


class JobResult(C.Structure):
    _fields_ = [("state", _i32), ("status", _i32), ("stats", Stats), ("rounds", _i32),
                ("submit_ms", C.c_double), ("admit_ms", C.c_double), ("done_ms", C.c_double),
                ("updates", C.c_double), ("device_bytes", C.c_uint64), ("tag", C.c_uint64),
                ("message", C.c_char * 128)]


class ServerInfo(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("queued", C.c_uint64), ("running", C.c_uint64), ("budget_bytes", C.c_uint64),
                ("bytes_in_use", C.c_uint64), ("bytes_peak", C.c_uint64), ("rounds", C.c_uint64),
                ("bp_launches", C.c_uint64), ("updates_done", C.c_double),
                ("oom_requeues", C.c_uint64), ("gpu_round_ms", C.c_double),
                ("host_round_ms", C.c_double), ("host_admit_ms", C.c_double)]


JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}
FAULT_ALLOC, FAULT_ADMIT = 1, 2


class TiltGpuError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"tiltgpu error {code} ({STATUS.get(code, '?')}): {msg}")


EXPORTS = {
    # name: (restype, argtypes)
    "tg_abi_version": (C.c_int, []),
    "tg_status_string": (C.c_char_p, [C.c_int]),
    "tg_last_error": (C.c_char_p, []),
    "tg_options_default": (None, [C.POINTER(Options)]),
    "tg_session_create": (C.c_int, [C.POINTER(Geometry), C.POINTER(Options), C.POINTER(_P)]),
    "tg_upload_projections": (C.c_int, [_P, _P, C.c_size_t]),
    "tg_set_projections_device": (C.c_int, [_P, _P, C.c_size_t]),
    "tg_reconstruct": (C.c_int, [_P]),
    "tg_synchronize": (C.c_int, [_P]),
    "tg_download_slices": (C.c_int, [_P, _i32, _i32, _P, C.POINTER(Stats)]),
    "tg_get_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "tg_download_slices_async": (C.c_int, [_P, _i32, _i32, _P]),
    "tg_volume_device": (_P, [_P]),
    "tg_session_last_run": (C.c_int, [_P, C.POINTER(RunInfo)]),
    "tg_session_dims": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
    "tg_session_device_bytes": (C.c_size_t, [_P]),
    "tg_session_destroy": (C.c_int, [_P]),
    "tg_session_set_stream": (C.c_int, [_P, _P]),
    "tg_batch_create": (C.c_int, [_i32, C.POINTER(_P)]),
    "tg_batch_add": (C.c_int, [_P, _P]),
    "tg_batch_clear": (C.c_int, [_P]),
    "tg_batch_reconstruct": (C.c_int, [_P]),
    "tg_batch_synchronize": (C.c_int, [_P]),
    "tg_batch_last_run": (C.c_int, [_P, C.POINTER(RunInfo)]),
    "tg_batch_destroy": (C.c_int, [_P]),
    "tg_gpu_session_new": (C.c_int, [_P, _P, C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t,
                                     C.c_size_t, _i32, C.POINTER(_P)]),
    "tg_gpu_session_reconstruct_row": (C.c_int, [_P, C.c_size_t, _P]),
    "tg_gpu_session_free": (None, [_P]),
    "tg_apply_rweighting": (C.c_int, [_P, C.c_size_t, C.c_size_t, C.c_size_t, _f, _f, _i32,
                                      _i32, _i32]),
    "tg_synth_projections": (C.c_int, [C.POINTER(PhantomSpec), _P, _P, _i32, _i32]),
    "tg_apply_rweighting_device_noalloc": (C.c_int, [_P, C.c_size_t, C.c_size_t, C.c_size_t, _f, _f,
                                                     _i32, _i32, _i32, _P]),
    "tg_studio_reconstruct": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, _i32]),
    "tg_ctf_options_default": (None, [C.POINTER(CtfOptions)]),
    "tg_ctf_strip_width": (C.c_int, [C.POINTER(CtfOptions), _i32, _P, _i32, C.POINTER(_i32)]),
    "tg_ctf_phaseflip": (C.c_int, [C.POINTER(CtfOptions), _P, _i32, _i32, _i32, _P, _i32, _P, _i32, _P,
                                   C.POINTER(Stats)]),
    "tg_ctf_correct_strip": (C.c_int, [_P, _P, C.POINTER(CtfStripParams), _i32]),
    "tg_upload_sections": (C.c_int, [_P, _i32, _i32, _P]),
    "tg_session_inject_wait_fault": (C.c_int, [_P, _i32, C.c_uint32]),
    "tg_session_view_sums": (C.c_int, [_P, _P]),
    "tg_sirt_begin": (C.c_int, [_P]),
    "tg_sirt_iterate": (C.c_int, [_P, _i32]),
    "tg_sirt_end": (C.c_int, [_P]),
    "tg_sirt_save": (C.c_int, [_P, _P, C.POINTER(_i32)]),
    "tg_sirt_restore": (C.c_int, [_P, _P, _i32]),
    "tg_session_set_view_means": (C.c_int, [_P, _P]),
    "tg_download_slices_f16_async": (C.c_int, [_P, _i32, _i32, _P]),
    "tg_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(_P)]),
    "tg_host_free": (C.c_int, [_P]),
    "tg_mrc_header_new": (C.c_int, [_i32, _i32, _i32, _i32, C.c_char_p, _P]),
    "tg_mrc_read": (C.c_int, [C.c_char_p, C.POINTER(MrcInfo), _i32, _i32, _P]),
    "tg_mrc_write_f32": (C.c_int, [C.c_char_p, _P, _P, _i32, _f, _f, _f]),
    "tg_tilt_output_header": (C.c_int, [_P, _i32, _i32, _P]),
    "tg_read_tilt_file": (C.c_int, [C.c_char_p, _P, _i32, C.POINTER(_i32)]),
    "tg_write_tilt_file": (C.c_int, [C.c_char_p, _P, _i32]),
    "tg_server_create": (C.c_int, [_i32, C.c_uint64, _i32, C.POINTER(_P)]),
    "tg_server_submit": (C.c_int, [_P, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "tg_server_poll": (C.c_int, [_P, C.c_uint64, C.POINTER(JobResult)]),
    "tg_server_wait": (C.c_int, [_P, C.c_uint64, _i32, C.POINTER(JobResult)]),
    "tg_server_release": (C.c_int, [_P, C.c_uint64]),
    "tg_server_get_info": (C.c_int, [_P, C.POINTER(ServerInfo)]),
    "tg_server_inject": (C.c_int, [_P, _i32, _i32]),
    "tg_server_destroy": (C.c_int, [_P]),
    "tg_submit": (C.c_int, [_P, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "tg_poll": (C.c_int, [_P, C.c_uint64, C.POINTER(JobResult)]),
}
# library-internal helpers exported for tests and the benchmark (not in the header)
EXTRA = {
    "tg_session_kernel_info": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32),
                                         C.POINTER(_i32), C.POINTER(_i32)]),
    "tg_session_set_variant": (C.c_int, [_P, _i32]),
    "tg_variant_name": (C.c_char_p, [_i32]),
    "tg_batch_plan_info": (C.c_int, [_P, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
}

_lib = None


def build(force=False):
    """Compile libtiltgpu.so and bin/tilt with nvcc (cross-compiles without a GPU)."""
    cmd = ["make", "-C", _HERE, "-j8"] + (["-B"] if force else [])
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is not built; run build() (make -C imod-rs_b200)")
        _lib = C.CDLL(LIB_PATH)
        for name, (res, args) in {**EXPORTS, **EXTRA}.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def check(rc):
    if rc != TG_OK:
        raise TiltGpuError(rc, lib().tg_last_error().decode(errors="replace"))


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _fptr(a):
    return None if a is None else a.ctypes.data_as(_fp)


def make_options(*, radial=(0.35, 0.05), hamming=False, exact_filter_size=None, no_weight=False,
                 fill_mode="mean", no_cosine_stretch=False, cosine_interp="linear",
                 max_cosine_tilt=80.0, log=False, sirt=0, sirt_relax=1.0, fake_sirt=0,
                 densweight=1.0, outscale=1.0, outadd=0.0, gpu=False, storage="fp32", device=0,
                 use_graphs=True, exact_xtilt=False) -> Options:
    o = Options()
    lib().tg_options_default(C.byref(o))
    o.radial_cutoff, o.radial_falloff = float(radial[0]), float(radial[1])
    o.hamming = int(bool(hamming))
    o.exact_filter_size = int(exact_filter_size or 0)
    o.no_weight = int(bool(no_weight))
    o.fill_mode = FILL.get(str(fill_mode).lower(), 0)
    o.no_cosine_stretch = int(bool(no_cosine_stretch))
    o.cosine_cubic = int(str(cosine_interp).lower() == "cubic")
    o.max_cosine_tilt = float(max_cosine_tilt)
    o.log_transform = int(bool(log))
    o.sirt_iters, o.sirt_relax, o.fake_sirt = int(sirt), float(sirt_relax), int(fake_sirt)
    o.densweight, o.outscale, o.outadd = float(densweight), float(outscale), float(outadd)
    o.gpu_compat = int(bool(gpu))
    o.storage = STORAGE[storage] if isinstance(storage, str) else int(storage)
    o.device, o.use_graphs = int(device), int(bool(use_graphs))
    o.exact_xtilt = int(bool(exact_xtilt))
    return o


class Session:
    """One tilt series resident on the device (tg_session_*)."""

    def __init__(self, nx, ny, nz, angles, *, width=None, thickness=0, xtilt=None, zfactor=None,
                 local=None, **opts):
        self._keep = [_f32(angles), _f32(xtilt), _f32(zfactor),
                      None if local is None else _f32(np.asarray(local).reshape(-1, 5))]
        ang, xt, zf, loc = self._keep
        g = Geometry()
        g.nx, g.ny, g.nz = int(nx), int(ny), int(nz)
        g.out_nx = int(width or 0)
        g.out_nz = int(thickness or 0)
        g.n_angles, g.angles = len(ang), _fptr(ang)
        if xt is not None:
            g.n_xtilt, g.xtilt = len(xt), _fptr(xt)
        if zf is not None:
            g.n_zfactor, g.zfactor = len(zf), _fptr(zf)
        if loc is not None:
            g.n_local, g.local, g.has_local = len(loc), _fptr(loc), 1
        self.opts = make_options(**opts)
        self.h = _P()
        check(lib().tg_session_create(C.byref(g), C.byref(self.opts), C.byref(self.h)))
        onx, onz, ony = _i32(), _i32(), _i32()
        check(lib().tg_session_dims(self.h, C.byref(onx), C.byref(onz), C.byref(ony)))
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.out_shape = (ony.value, onz.value, onx.value)

    def upload(self, proj):
        p = _f32(proj)
        check(lib().tg_upload_projections(self.h, _ptr(p), p.size))

    def set_device(self, dev_ptr: int, n: int):
        check(lib().tg_set_projections_device(self.h, _P(dev_ptr), n))

    def reconstruct(self, sync=True):
        check(lib().tg_reconstruct(self.h))
        if sync:
            check(lib().tg_synchronize(self.h))

    def synchronize(self):
        check(lib().tg_synchronize(self.h))

    def download(self, y0=0, y1=None, out=None):
        y1 = self.out_shape[0] if y1 is None else y1
        shape = (y1 - y0,) + self.out_shape[1:]
        if out is None:
            out = np.empty(shape, np.float32)
        st = Stats()
        check(lib().tg_download_slices(self.h, y0, y1, _ptr(out), C.byref(st)))
        return out, {"amin": st.amin, "amax": st.amax, "amean": st.amean}

    def stats(self):
        st = Stats()
        check(lib().tg_get_stats(self.h, C.byref(st)))
        return {"amin": st.amin, "amax": st.amax, "amean": st.amean}

    def volume_ptr(self) -> int:
        return lib().tg_volume_device(self.h)

    def last_run(self):
        ri = RunInfo()
        check(lib().tg_session_last_run(self.h, C.byref(ri)))
        return {k: getattr(ri, k) for k, _ in RunInfo._fields_}

    def kernel_info(self):
        vals = [_i32() for _ in range(5)]
        check(lib().tg_session_kernel_info(self.h, *[C.byref(v) for v in vals]))
        fast, variant, fmt, padl, pw = (v.value for v in vals)
        name = {2: "xtilt-staged"}.get(fast, "general")
        if fast in (1, 3):
            name = lib().tg_variant_name(variant).decode() + ("+xtilt-blend" if fast == 3 else "")
        return {"fast": fast == 1, "xtilt_split": fast == 3, "variant": variant,
                "variant_name": name, "fmt": fmt, "padL": padl, "PW": pw}

    def view_sums(self):
        """Per-view f64 sums of the uploaded rows (after --log), for slab sharding."""
        out = np.empty(self.nz, np.float64)
        check(lib().tg_session_view_sums(self.h, _ptr(out)))
        return out

    def set_view_means(self, means):
        """Pins the mean fill values (whole-series means of a slab); None: compute them again."""
        m = None if means is None else _f32(means)
        check(lib().tg_session_set_view_means(self.h, _ptr(m)))

    # SIRT in steps with checkpoints (tg_sirt_*)
    def sirt_begin(self):
        """Log, means, R-weighting and the WBP start; 0 SIRT iterations done."""
        check(lib().tg_sirt_begin(self.h))

    def sirt_iterate(self, n: int):
        check(lib().tg_sirt_iterate(self.h, int(n)))

    def sirt_end(self):
        """Output stage: the volume and statistics of tg_reconstruct with the iterations run."""
        check(lib().tg_sirt_end(self.h))

    def sirt_save(self):
        """(raw SIRT volume [y][z][x], iterations done), synchronising."""
        vol = np.empty(self.out_shape, np.float32)
        done = _i32(0)
        check(lib().tg_sirt_save(self.h, _ptr(vol), C.byref(done)))
        return vol, int(done.value)

    def sirt_restore(self, vol, iterations_done: int):
        v = np.ascontiguousarray(vol, np.float32)
        if v.shape != tuple(self.out_shape):
            raise ValueError(f"volume shape {v.shape} != {tuple(self.out_shape)}")
        check(lib().tg_sirt_restore(self.h, _ptr(v), int(iterations_done)))

    def inject_wait_fault(self, skip_stage=-1, wait_limit_us=0):
        """Test hook: the back-projector's producer leaves out one pipeline stage and
        its bounded waits give up after wait_limit_us (see tiltgpu.h)."""
        check(lib().tg_session_inject_wait_fault(self.h, int(skip_stage), int(wait_limit_us)))

    def set_variant(self, v: int):
        check(lib().tg_session_set_variant(self.h, v))

    def set_stream(self, stream_handle: int):
        """Run on the caller's cudaStream_t (an integer handle; 0 = own stream)."""
        check(lib().tg_session_set_stream(self.h, _P(stream_handle or None)))

    def device_bytes(self):
        return lib().tg_session_device_bytes(self.h)

    def close(self):
        if self.h:
            lib().tg_session_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Many sessions reconstructed together (tg_batch_*): one persistent
    back-projection launch per round across all fast-path series."""

    def __init__(self, device=0):
        self.h = _P()
        check(lib().tg_batch_create(device, C.byref(self.h)))
        self.sessions = []

    def add(self, s: "Session"):
        check(lib().tg_batch_add(self.h, s.h))
        self.sessions.append(s)

    def clear(self):
        check(lib().tg_batch_clear(self.h))
        self.sessions = []

    def reconstruct(self, sync=True):
        check(lib().tg_batch_reconstruct(self.h))
        if sync:
            self.synchronize()

    def synchronize(self):
        check(lib().tg_batch_synchronize(self.h))

    def last_run(self):
        ri = RunInfo()
        check(lib().tg_batch_last_run(self.h, C.byref(ri)))
        return {k: getattr(ri, k) for k, _ in RunInfo._fields_}

    def plan_info(self):
        """SIRT rounds of the last reconstruction: rounds replayed from a CUDA graph,
        grouped reprojection / filter launches and kernels per round."""
        v = [_i32() for _ in range(4)]
        check(lib().tg_batch_plan_info(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("graph_rounds", "fp_groups", "filter_groups", "round_launches"), (x.value for x in v)))

    def close(self):
        if self.h:
            lib().tg_batch_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _geometry(nx, ny, nz, angles, width, thickness, xtilt, zfactor, local, keep):
    ang, xt, zf = _f32(angles), _f32(xtilt), _f32(zfactor)
    loc = None if local is None else _f32(np.asarray(local).reshape(-1, 5))
    keep += [ang, xt, zf, loc]
    g = Geometry()
    g.nx, g.ny, g.nz = int(nx), int(ny), int(nz)
    g.out_nx = int(width or 0)
    g.out_nz = int(thickness or 0)
    g.n_angles, g.angles = len(ang), _fptr(ang)
    if xt is not None:
        g.n_xtilt, g.xtilt = len(xt), _fptr(xt)
    if zf is not None:
        g.n_zfactor, g.zfactor = len(zf), _fptr(zf)
    if loc is not None:
        g.n_local, g.local, g.has_local = len(loc), _fptr(loc), 1
    return g


def _result(r: JobResult):
    return {"state": JOB_STATES.get(r.state, r.state), "status": r.status,
            "stats": {"amin": r.stats.amin, "amax": r.stats.amax, "amean": r.stats.amean},
            "rounds": r.rounds, "submit_ms": r.submit_ms, "admit_ms": r.admit_ms,
            "done_ms": r.done_ms, "updates": r.updates, "device_bytes": r.device_bytes,
            "tag": r.tag, "message": r.message.decode(errors="replace")}


class Server:
    """Request loop with continuous batching (tg_server_*).  Jobs are submitted
    from any thread; their projection arrays (and output arrays) are kept alive
    here until the job is released."""

    def __init__(self, device=0, budget_bytes=0, max_active=64):
        self.h = _P()
        check(lib().tg_server_create(device, int(budget_bytes), int(max_active), C.byref(self.h)))
        self._keep = {}

    def submit(self, proj, angles, *, out=None, width=None, thickness=0, xtilt=None, zfactor=None,
               local=None, tag=0, **opts):
        """proj: float32 (nz, ny, nx) host array (pinned memory copies fastest);
        out: float32 host array of the output volume (ny, thickness, width) or None."""
        nz, ny, nx = proj.shape
        keep = [proj, out]
        p = proj if (proj.dtype == np.float32 and proj.flags.c_contiguous) else _f32(proj)
        keep.append(p)
        if out is not None and not (out.dtype == np.float32 and out.flags.c_contiguous and out.flags.writeable):
            raise ValueError("out must be a writeable C-contiguous float32 array")
        j = Job()
        j.geometry = _geometry(nx, ny, nz, angles, width, thickness, xtilt, zfactor, local, keep)
        j.options = make_options(**opts)
        j.projections = p.ctypes.data
        j.n_projections = p.size
        j.volume_out = None if out is None else out.ctypes.data
        j.tag = int(tag)
        jid = C.c_uint64()
        check(lib().tg_server_submit(self.h, C.byref(j), C.byref(jid)))
        self._keep[jid.value] = keep
        return jid.value

    def poll(self, jid):
        r = JobResult()
        check(lib().tg_server_poll(self.h, jid, C.byref(r)))
        return _result(r)

    def wait(self, jid, timeout_ms=-1):
        r = JobResult()
        rc = lib().tg_server_wait(self.h, jid, int(timeout_ms), C.byref(r))
        if rc == -9:
            return None
        check(rc)
        return _result(r)

    def release(self, jid):
        check(lib().tg_server_release(self.h, jid))
        self._keep.pop(jid, None)

    def info(self):
        i = ServerInfo()
        check(lib().tg_server_get_info(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in ServerInfo._fields_}

    def inject(self, fault, count=1):
        check(lib().tg_server_inject(self.h, int(fault), int(count)))

    def close(self):
        if self.h:
            lib().tg_server_destroy(self.h)
            self.h = _P()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def reconstruct(proj, angles, **kw):
    """One-shot: upload, reconstruct, download.  Returns (volume, stats)."""
    nz, ny, nx = proj.shape
    with Session(nx, ny, nz, angles, **kw) as s:
        s.upload(proj)
        s.reconstruct()
        return s.download()


class GpuSession:
    """GpuSession::new / reconstruct_row of apps/tilt/src/gpu.rs, on the B200 kernels."""

    def __init__(self, projections, tilt_cos_sin, in_nx, in_ny, n_projs, out_nx, out_nz, device=0):
        self._p = _f32(projections)
        self._cs = _f32(np.asarray(tilt_cos_sin).reshape(-1, 2))
        self.out = (out_nz, out_nx)
        self.h = _P()
        check(lib().tg_gpu_session_new(_ptr(self._p), _ptr(self._cs), in_nx, in_ny, n_projs, out_nx,
                                       out_nz, device, C.byref(self.h)))

    def reconstruct_row(self, iy):
        out = np.empty(self.out, np.float32)
        check(lib().tg_gpu_session_reconstruct_row(self.h, iy, _ptr(out)))
        return out

    def close(self):
        if self.h:
            lib().tg_gpu_session_free(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def apply_rweighting(proj, cutoff=0.35, falloff=0.05, exact_filter_size=None, use_hamming=False,
                     device=0):
    """apply_rweighting (apps/tilt/src/main.rs:333) on the device; returns a new array."""
    p = np.array(proj, dtype=np.float32, copy=True, order="C")
    nz, ny, nx = p.shape
    check(lib().tg_apply_rweighting(_ptr(p), nx, ny, nz, cutoff, falloff, int(exact_filter_size or 0),
                                    int(use_hamming), device))
    return p


def apply_rweighting_device_noalloc(dev_ptr: int, nx, ny, nz, cutoff=0.35, falloff=0.05,
                                    exact_filter_size=None, use_hamming=False, device=0, stream=0):
    """In-place R-weighting of a device stack without any device allocation."""
    check(lib().tg_apply_rweighting_device_noalloc(_P(dev_ptr), nx, ny, nz, cutoff, falloff,
                                                   int(exact_filter_size or 0), int(use_hamming),
                                                   device, _P(stream or None)))


def studio_reconstruct(ali_path, tlt_path, rec_path, device=0):
    """imod-studio's reconstruction step (apps/imod-studio/src/main.rs:725-776) on the GPU."""
    check(lib().tg_studio_reconstruct(str(ali_path).encode(), str(tlt_path).encode(), str(rec_path).encode(),
                                      device))


def ctf_options(**kw):
    """tg_ctf_options with the reference's defaults (apps/ctfphaseflip/src/main.rs:19-88)."""
    o = CtfOptions()
    lib().tg_ctf_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def ctf_phaseflip(stack, angles, view_defocus=None, **kw):
    """CTF phase flip of a [nz][ny][nx] stack on the GPU.  Returns (out, stats)."""
    st_in = _f32(stack)
    nz, ny, nx = st_in.shape
    a = _f32(angles)
    vd = None if view_defocus is None else _f32(np.asarray(view_defocus).reshape(-1, 3))
    o = ctf_options(**kw)
    out = np.empty_like(st_in)
    st = Stats()
    check(lib().tg_ctf_phaseflip(C.byref(o), _ptr(st_in), nx, ny, nz, _ptr(a), len(a), _ptr(vd),
                                 0 if vd is None else len(vd), _ptr(out), C.byref(st)))
    return out, {"amin": st.amin, "amax": st.amax, "amean": st.amean}


def ctf_strip_width(nx, view_defocus=None, **kw):
    vd = None if view_defocus is None else _f32(np.asarray(view_defocus).reshape(-1, 3))
    o = ctf_options(**kw)
    w = _i32()
    check(lib().tg_ctf_strip_width(C.byref(o), nx, _ptr(vd), 0 if vd is None else len(vd), C.byref(w)))
    return w.value


def ctf_correct_strip(re, im, device=0, **params):
    """GpuCtfSession::correct_strip on one strip's 2D FFT (re, im: sw*sh floats); copies returned."""
    r = np.array(re, dtype=np.float32, copy=True, order="C")
    i = np.array(im, dtype=np.float32, copy=True, order="C")
    p = CtfStripParams(**params)
    check(lib().tg_ctf_correct_strip(_ptr(r), _ptr(i), C.byref(p), device))
    return r, i


def synth_projections(angles, *, nx, ny, vol_nx=None, vol_nz, n_ell=300, rmin=3.0, rmax=40.0,
                      dmin=0.2, dmax=1.0, n_beads=40, bead_r=5.0, bead_d=5.0, noise_kind=1,
                      noise=0.5, xtilt_deg=0.0, seed=1, device=0, out_device_ptr=None):
    """Seeded phantom projections [nz][ny][nx] (host array, or into a device pointer)."""
    ang = _f32(angles)
    sp = PhantomSpec()
    sp.seed, sp.nx, sp.ny, sp.nz = int(seed), int(nx), int(ny), len(ang)
    sp.vol_nx, sp.vol_nz = int(vol_nx or nx), int(vol_nz)
    sp.n_ell, sp.rmin, sp.rmax, sp.dmin, sp.dmax = int(n_ell), rmin, rmax, dmin, dmax
    sp.n_beads, sp.bead_r, sp.bead_d = int(n_beads), bead_r, bead_d
    sp.noise_kind, sp.noise, sp.xtilt_deg = int(noise_kind), noise, xtilt_deg
    if out_device_ptr is not None:
        check(lib().tg_synth_projections(C.byref(sp), _ptr(ang), _P(out_device_ptr), 1, device))
        return None
    out = np.empty((len(ang), ny, nx), np.float32)
    check(lib().tg_synth_projections(C.byref(sp), _ptr(ang), _ptr(out), 0, device))
    return out


# ---- MRC / tilt-file boundary (host only) ----
MODES = {"Byte": 0, "Short": 1, "Float": 2, "ComplexShort": 3, "ComplexFloat": 4, "UShort": 6,
         "HalfFloat": 12, "Rgb": 16, "FourBit": 101}


def mrc_header_new(nx, ny, nz, mode, label=None) -> bytes:
    buf = (C.c_uint8 * 1024)()
    check(lib().tg_mrc_header_new(nx, ny, nz, MODES.get(mode, mode) if isinstance(mode, str) else mode,
                                  None if label is None else label.encode(), buf))
    return bytes(buf)


def mrc_info(path):
    info = MrcInfo()
    check(lib().tg_mrc_read(str(path).encode(), C.byref(info), 0, 0, None))
    return info


def mrc_read(path, z0=0, z1=None, values_per_section=None):
    info = mrc_info(path)
    z1 = info.nz if z1 is None else z1
    per = values_per_section or info.nx * info.ny * (3 if info.mode == 16 else 1)
    out = np.empty((z1 - z0) * per, np.float32)
    check(lib().tg_mrc_read(str(path).encode(), None, z0, z1, _ptr(out)))
    return info, out


def mrc_write_f32(path, header: bytes, data, stats=(0.0, 0.0, 0.0)):
    hb = (C.c_uint8 * 1024).from_buffer_copy(header)
    d = _f32(data)
    nx, ny = np.frombuffer(header[:8], "<i4")
    nsec = d.size // int(nx * ny) if d is not None else 0
    check(lib().tg_mrc_write_f32(str(path).encode(), hb, _ptr(d), nsec, *stats))


def tilt_output_header(in_header: bytes, out_nx, out_nz) -> bytes:
    hin = (C.c_uint8 * 1024).from_buffer_copy(in_header)
    out = (C.c_uint8 * 1024)()
    check(lib().tg_tilt_output_header(hin, out_nx, out_nz, out))
    return bytes(out)


def read_tilt_file(path, cap=100000):
    out = np.empty(cap, np.float32)
    n = _i32()
    check(lib().tg_read_tilt_file(str(path).encode(), _ptr(out), cap, C.byref(n)))
    return out[:min(n.value, cap)].copy()


def write_tilt_file(path, angles):
    a = _f32(angles)
    check(lib().tg_write_tilt_file(str(path).encode(), _ptr(a), len(a)))
