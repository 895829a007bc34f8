"""Hilbert spectral analysis of IMFs (hilbert.py) against scipy.signal on CPU, and the CUDA
path against the CPU path."""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _hilbert_mod():
    spec = importlib.util.spec_from_file_location(
        "hilbert_mod", os.path.join(ROOT, "ceemdan-gpu_b200", "hilbert.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("n", [1, 2, 7, 256, 1001, 4096])
def test_analytic_matches_scipy(n):
    import torch
    from scipy.signal import hilbert
    hb = _hilbert_mod()
    x = np.random.default_rng(n).standard_normal((3, n))
    z = hb.analytic(torch.tensor(x)).numpy()
    ref = hilbert(x, axis=-1)
    assert np.max(np.abs(z - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
    z1 = hb.analytic(torch.tensor(x[0])).numpy()
    assert np.array_equal(z1, z[0])


def test_phase_unwraps_like_numpy_and_frequency_of_a_tone():
    import torch
    hb = _hilbert_mod()
    fs, f0, n = 256.0, 10.0, 4096
    t = np.arange(n) / fs
    x = np.stack([np.cos(2 * np.pi * f0 * t), 0.5 * np.sin(2 * np.pi * 3.0 * t)])
    ph = hb.phase(torch.tensor(x)).numpy()
    z = hb.analytic(torch.tensor(x)).numpy()
    assert np.max(np.abs(ph - np.unwrap(np.angle(z), axis=-1))) <= 1e-9
    fr = hb.inst_frequency(torch.tensor(x), fs).numpy()
    mid = slice(n // 8, -n // 8)  # away from the edge effects of the FFT definition
    assert np.max(np.abs(fr[0, mid] - f0)) < 1e-6
    assert np.max(np.abs(fr[1, mid] - 3.0)) < 1e-6
    amp = hb.amplitude(torch.tensor(x)).numpy()
    assert np.max(np.abs(amp[0, mid] - 1.0)) < 1e-9
    assert np.max(np.abs(amp[1, mid] - 0.5)) < 1e-9


def test_float32_keeps_single_precision():
    import torch
    hb = _hilbert_mod()
    x = torch.tensor(np.random.default_rng(0).standard_normal(512), dtype=torch.float32)
    assert hb.analytic(x).dtype == torch.complex64


@pytest.mark.gpu
def test_cuda_matches_cpu_on_imfs(pkg, cuda, wl):
    import torch
    hb = _hilbert_mod()
    x = wl.eeg_like(8192, seed=3)
    imfs = pkg.iceemdan(torch.tensor(x, device=cuda), 16, 6, 80, 0.2, noise_sift_cap=200)
    g = hb.inst_frequency(imfs, 256.0).cpu().numpy()
    c = hb.inst_frequency(imfs.cpu(), 256.0).numpy()
    assert np.max(np.abs(g - c)) <= 1e-9 * max(1.0, np.max(np.abs(c)))
    ga = hb.amplitude(imfs).cpu().numpy()
    ca = hb.amplitude(imfs.cpu()).numpy()
    assert np.max(np.abs(ga - ca)) <= 1e-12 * np.max(ca)
