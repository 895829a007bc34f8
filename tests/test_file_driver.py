"""ceemdan_file, the file-level driver (sample_binary_file.cu:36-83): raw float32 samples in,
raw num_IMFs x N float32 modes out.  CPU tests cover the argument and file checks, which end
before any GPU work; the GPU test compares the written modes with the tensor API."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "ceemdan-gpu_b200", "ceemdan_file")


@pytest.fixture(scope="module")
def exe(built_lib):
    if not os.path.exists(EXE):
        subprocess.run(["make", "-C", os.path.join(ROOT, "ceemdan-gpu_b200")], check=True,
                       capture_output=True)
    return EXE


def _run(exe, *args):
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)


def test_help_and_usage_errors(exe):
    r = _run(exe, "--help")
    assert r.returncode == 0 and "usage: ceemdan_file" in r.stdout
    assert _run(exe).returncode == 2
    assert _run(exe, "a.bin").returncode == 2
    assert _run(exe, "a.bin", "b.bin", "--nr").returncode == 2
    assert _run(exe, "a.bin", "b.bin", "--imfs", "1").returncode == 2
    assert _run(exe, "a.bin", "b.bin", "--nr", "-3").returncode == 2
    assert _run(exe, "a.bin", "b.bin", "--bogus").returncode == 2


def test_input_errors_end_before_gpu_work(exe, tmp_path):
    r = _run(exe, tmp_path / "missing.bin", tmp_path / "out.bin")
    assert r.returncode == 1 and "cannot read" in r.stderr
    bad = tmp_path / "odd.bin"
    bad.write_bytes(b"\x00" * 10)  # not a whole number of float32 samples
    r = _run(exe, bad, tmp_path / "out.bin")
    assert r.returncode == 1 and "whole number" in r.stderr
    short = tmp_path / "short.bin"
    np.zeros(3, dtype=np.float32).tofile(short)
    r = _run(exe, short, tmp_path / "out.bin")
    assert r.returncode == 1 and "fewer than 4" in r.stderr
    ok = tmp_path / "ok.bin"
    np.zeros(64, dtype=np.float32).tofile(ok)
    r = _run(exe, ok, tmp_path / "no_such_dir" / "out.bin")
    assert r.returncode == 1 and "cannot write" in r.stderr


@pytest.mark.gpu
def test_modes_file_matches_tensor_api(exe, pkg, cuda, wl, tmp_path):
    import torch
    n, nr, nimf, mi = 3000, 8, 5, 60
    x = wl.eeg_like(n, seed=9).astype(np.float32)
    src = tmp_path / "signal.bin"
    x.tofile(src)
    dst = tmp_path / "modes.bin"
    r = _run(exe, src, dst, "--nr", nr, "--imfs", nimf, "--max-iter", mi, "--noise-cap", 200)
    assert r.returncode == 0, r.stderr
    assert "Execution time:" in r.stdout
    modes = np.fromfile(dst, dtype=np.float32).reshape(nimf, n)
    ref = pkg.iceemdan(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2, seed=1234,
                       noise_sift_cap=200).cpu().numpy()
    assert np.array_equal(modes, ref)
    # --f64: float64 file in and out, iceemdanD semantics
    x64 = x.astype(np.float64)
    src64 = tmp_path / "signal64.bin"
    x64.tofile(src64)
    dst64 = tmp_path / "modes64.bin"
    r = _run(exe, src64, dst64, "--f64", "--nr", nr, "--imfs", nimf, "--max-iter", mi,
             "--noise-cap", 200, "--seed", 7)
    assert r.returncode == 0, r.stderr
    ref64 = pkg.iceemdan(torch.tensor(x64, device=cuda), nr, nimf, mi, 0.2, seed=7,
                         noise_sift_cap=200).cpu().numpy()
    assert np.array_equal(np.fromfile(dst64, dtype=np.float64).reshape(nimf, n), ref64)
