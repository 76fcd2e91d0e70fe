"""Host logic of the drop-in `ctfphaseflip` CLI (apps/ctfphaseflip/src/main.rs:
19-88 flags, 94-209 defocus file, 221-240 errors and exit codes).  No GPU."""
import subprocess

import numpy as np
import pytest

import tiltgpu as T


def run(*args):
    return subprocess.run([T.CTF_CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=60)


def write_inputs(tmp_path, nz=3):
    src, tlt = tmp_path / "in.mrc", tmp_path / "in.tlt"
    T.mrc_write_f32(src, T.mrc_header_new(16, 8, nz, "Float"), np.ones((nz, 8, 16), np.float32))
    T.write_tilt_file(tlt, np.zeros(nz, np.float32))
    return src, tlt


def test_help_lists_the_reference_flags():
    r = run("--help")
    assert r.returncode == 0
    for f in ("--defocus-file", "--strip-width", "--tilt-axis-angle", "--max-strip-width",
              "--amplitude-contrast", "--cuton-freq", "--plate-phase", "--pixel-size", "--voltage", "--cs"):
        assert f in r.stdout


def test_missing_and_bad_arguments():
    r = run("-i", "a.mrc")
    assert r.returncode == 2 and "--output" in r.stderr and "--tilt-file" in r.stderr
    assert run("-i", "a", "-o", "b", "-t", "c", "-w", "x").returncode == 2
    assert run("-i", "a", "-o", "b", "-t", "c", "--gpu=1").returncode == 2
    assert run("-i", "a", "-o", "b", "-t", "c", "--bogus", "1").returncode == 2


def test_unreadable_tilt_file_and_mrc(tmp_path):
    r = run("-i", tmp_path / "no.mrc", "-o", tmp_path / "o.mrc", "-t", tmp_path / "no.tlt")
    assert r.returncode == 1 and "Error reading tilt file" in r.stderr
    src, tlt = write_inputs(tmp_path)
    r = run("-i", tmp_path / "no.mrc", "-o", tmp_path / "o.mrc", "-t", tlt)
    assert r.returncode == 1 and "Error" in r.stderr


@pytest.mark.parametrize("content,msg", [
    ("0 -2000\n1\n", "line 2: expected at least 'view defocus1'"),
    ("x -2000\n", "invalid view number 'x'"),
    ("0 abc\n", "invalid defocus1 'abc'"),
    ("0 -2000 q 3\n", "invalid defocus2 'q'"),
    ("0 -2000 -2100 z\n", "invalid astig_angle 'z'"),
])
def test_defocus_file_errors(tmp_path, content, msg):
    src, tlt = write_inputs(tmp_path)
    df = tmp_path / "d.txt"
    df.write_text(content)
    r = run("-i", src, "-o", tmp_path / "o.mrc", "-t", tlt, "--defocus-file", df)
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_no_gpu_is_an_error_not_a_fallback(tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    src, tlt = write_inputs(tmp_path)
    r = run("-i", src, "-o", tmp_path / "o.mrc", "-t", tlt, "-p", "2")
    assert r.returncode == 1 and "no" in r.stderr.lower()
