"""Host logic of the drop-in `tilt` CLI: flags, errors and exit codes
(apps/tilt/src/main.rs:18-120, 550-558, 656-680).  No GPU needed."""
import os
import subprocess

import numpy as np
import pytest

import tiltgpu as T


def run(*args):
    return subprocess.run([T.CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=60)


def test_help():
    r = run("--help")
    assert r.returncode == 0 and "--tilt-file" in r.stdout and "--fake-sirt" in r.stdout


def test_exact_xtilt_flag():
    r = run("--help")
    assert "--exact-xtilt" in r.stdout
    # a flag takes no value
    r = run("-i", "a", "-o", "b", "-t", "c", "--exact-xtilt=1")
    assert r.returncode == 2 and "exact-xtilt" in r.stderr


def test_missing_required_arguments():
    r = run("-i", "a.mrc")
    assert r.returncode == 2 and "--output" in r.stderr and "--tilt-file" in r.stderr


def test_bad_numeric_value():
    r = run("-i", "a", "-o", "b", "-t", "c", "--sirt", "x")
    assert r.returncode == 2 and "invalid value" in r.stderr
    r = run("-i", "a", "-o", "b", "-t", "c", "--no-weight=1")
    assert r.returncode == 2


def test_unreadable_tilt_file(tmp_path):
    r = run("-i", tmp_path / "in.mrc", "-o", tmp_path / "o.mrc", "-t", tmp_path / "none.tlt")
    assert r.returncode == 1 and r.stderr.startswith("Error reading tilt file:")


def test_unreadable_mrc(tmp_path):
    t = tmp_path / "a.tlt"
    T.write_tilt_file(t, [0.0])
    r = run("-i", tmp_path / "none.mrc", "-o", tmp_path / "o.mrc", "-t", t)
    assert r.returncode == 1 and r.stderr.startswith("Error:")


def test_bad_xtilt_file(tmp_path):
    t = tmp_path / "a.tlt"
    T.write_tilt_file(t, [0.0, 5.0])
    m = tmp_path / "in.mrc"
    T.mrc_write_f32(m, T.mrc_header_new(8, 4, 2, "Float"), np.ones(64, np.float32))
    x = tmp_path / "x.txt"
    open(x, "w").write("1.0\nnot-a-number\n")
    r = run("-i", m, "-o", tmp_path / "o.mrc", "-t", t, "--xtilt-file", x)
    assert r.returncode == 1 and r.stderr.splitlines()[-1].startswith("Error reading xtilt file: parse error")


def test_pip_aliases_parse(tmp_path):
    # PIP-style keys map onto the same fields; with no tilt file readable the run stops there
    r = run("-InputProjections", "a", "-OutputFile", "b", "-TILTFILE", tmp_path / "none.tlt",
            "-THICKNESS", "100", "-RADIAL", "0.3,0.05", "-SIRTIterations", "3", "-LOG", "0.0",
            "-SCALE", "1.0,2.0")
    assert r.returncode == 1 and "Error reading tilt file" in r.stderr


def test_no_gpu_is_an_error_not_a_fallback(tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    t = tmp_path / "a.tlt"
    T.write_tilt_file(t, [0.0, 5.0])
    m = tmp_path / "in.mrc"
    T.mrc_write_f32(m, T.mrc_header_new(8, 4, 2, "Float"), np.ones(64, np.float32))
    r = run("-i", m, "-o", tmp_path / "o.mrc", "-t", t)
    assert r.returncode == 1 and "no sm_100 CUDA device" in r.stderr
    assert not os.path.exists(tmp_path / "o.mrc")


def test_mode_flag_accepts_2_and_12_only():
    r = run("-i", "a", "-o", "b", "-t", "c", "--mode", "4")
    assert r.returncode == 2 and "--mode" in r.stderr
    assert "--mode" in run("--help").stdout and "--io-chunk-kb" in run("--help").stdout


def test_checkpoint_flags():
    h = run("--help").stdout
    assert "--checkpoint <FILE>" in h and "--checkpoint-every" in h and "--resume <FILE>" in h
    r = run("-i", "a", "-o", "b", "-t", "c", "--checkpoint-every", "x")
    assert r.returncode == 2 and "--checkpoint-every" in r.stderr
    r = run("-i", "a", "-o", "b", "-t", "c", "--resume")
    assert r.returncode == 2 and "a value is required for '--resume'" in r.stderr
    r = run("-i", "a", "-o", "b", "-t", "c", "--resume", "s.mrc")
    assert r.returncode == 2 and "need SIRT iterations" in r.stderr
    r = run("-i", "a", "-o", "b", "-t", "c", "--sirt", "3", "--gpu", "--checkpoint", "s.mrc")
    assert r.returncode == 2 and "need SIRT iterations" in r.stderr
