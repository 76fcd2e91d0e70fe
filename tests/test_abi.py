"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import tiltgpu as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "tiltgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tg_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(T.LIB_PATH)
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) <= set(T.EXPORTS), set(declared()) - set(T.EXPORTS)


def test_abi_version_and_defaults():
    assert T.lib().tg_abi_version() == 1
    o = T.make_options()
    # apps/tilt/src/main.rs:18-120 defaults
    assert (o.radial_cutoff, o.radial_falloff) == (np.float32(0.35), np.float32(0.05))
    assert o.max_cosine_tilt == 80.0 and o.sirt_relax == 1.0 and o.fill_mode == 0
    assert (o.densweight, o.outscale, o.outadd) == (1.0, 1.0, 0.0)
    assert o.sirt_iters == 0 and o.fake_sirt == 0 and o.no_weight == 0
    assert T.lib().tg_status_string(-8) == b"input on which the reference panics"


def test_options_struct_matches_header():
    # tg_options_default clears the whole C struct: a sentinel right after the
    # Python mirror must survive (the mirror is not shorter than the C struct),
    # and the last field (exact_xtilt) defaults to 0 with use_graphs on
    n = C.sizeof(T.Options)
    buf = (C.c_ubyte * (n + 32))(*([0xA5] * (n + 32)))
    T.lib().tg_options_default(C.cast(buf, C.POINTER(T.Options)))
    assert bytes(buf[n:]) == b"\xa5" * 32
    o = T.Options.from_buffer_copy(bytes(buf[:n]))
    assert o.use_graphs == 1 and o.exact_xtilt == 0
    assert T.make_options(exact_xtilt=True).exact_xtilt == 1


def test_session_without_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(T.TiltGpuError) as e:
        T.Session(8, 2, 3, [0, 1, 2])
    assert e.value.code == -7


def test_invalid_arguments_rejected():
    with pytest.raises(T.TiltGpuError) as e:
        T.Session(1, 2, 3, [0, 1, 2])  # nx < 2
    assert e.value.code == -1
    with pytest.raises(T.TiltGpuError) as e:
        T.Session(8, 2, 3, [0, float("nan"), 2])
    assert e.value.code in (-1, -7)
