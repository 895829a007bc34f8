"""Seeded synthetic input signals for the decomposition workloads.

The reference ships no benchmark data beyond two EEG channels; the workloads it is measured
on are described by shape, length, sampling rate and content, and are generated here from
fixed seeds so that every run (GPU engine, CPU oracle, benchmark) sees identical inputs.
"""
from __future__ import annotations

import numpy as np

FS = 256.0


def two_tone_chirp(n: int = 4096, seed: int = 0, fs: float = FS) -> np.ndarray:
    """1.0*sin(2pi*5t) + 0.5*sin(2pi*40t) + 0.3*linear chirp 1->30 Hz + N(0, 0.1^2)."""
    rng = np.random.default_rng(seed)
    t = np.arange(n, dtype=np.float64) / fs
    t1 = n / fs
    chirp = np.cos(2.0 * np.pi * (1.0 * t + (30.0 - 1.0) / (2.0 * t1) * t * t))
    x = (np.sin(2.0 * np.pi * 5.0 * t) + 0.5 * np.sin(2.0 * np.pi * 40.0 * t)
         + 0.3 * chirp + 0.1 * rng.standard_normal(n))
    return x


def eeg_like(n: int = 244032, seed: int = 2, fs: float = FS, alpha_hz: float = 10.0) -> np.ndarray:
    """EEG-shaped channel: unit-variance 1/f noise + alpha bursts + beta + spikes.

    - 1/f ("pink") noise: N(0,1) shaped by 1/sqrt(f) in the Fourier domain, DC removed,
      rescaled to unit variance;
    - alpha bursts at ``alpha_hz``: Poisson onsets at 0.3/s, lengths U(0.5, 2) s, Gaussian
      envelope (sigma = length/6), amplitude 2;
    - 20 Hz beta rhythm, amplitude 0.5;
    - biphasic 50 ms spikes (one period of a 20 Hz sine), Poisson at 0.05/s, amplitude 5.
    """
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(n)
    spec = np.fft.rfft(w)
    f = np.fft.rfftfreq(n, d=1.0 / fs)
    scale = np.zeros_like(f)
    scale[1:] = 1.0 / np.sqrt(f[1:])
    pink = np.fft.irfft(spec * scale, n)
    pink = (pink - pink.mean()) / pink.std()
    t = np.arange(n, dtype=np.float64) / fs
    dur = n / fs
    x = pink + 0.5 * np.sin(2.0 * np.pi * 20.0 * t + rng.uniform(0, 2 * np.pi))
    for _ in range(rng.poisson(0.3 * dur)):
        t0 = rng.uniform(0.0, dur)
        ln = rng.uniform(0.5, 2.0)
        c = t0 + ln / 2.0
        env = np.exp(-0.5 * ((t - c) / (ln / 6.0)) ** 2)
        x += 2.0 * env * np.sin(2.0 * np.pi * alpha_hz * t + rng.uniform(0, 2 * np.pi))
    for _ in range(rng.poisson(0.05 * dur)):
        t0 = rng.uniform(0.0, dur)
        m = (t >= t0) & (t < t0 + 0.05)
        x[m] += 5.0 * np.sin(2.0 * np.pi * (t[m] - t0) / 0.05)
    return x


def white_noise(nr: int, n: int, seed: int = 1) -> np.ndarray:
    """NR x N float64 N(0,1) realizations (realization-major)."""
    return np.random.default_rng(seed).standard_normal((nr, n))


def ragged_batch(channels: int = 64, lo: int = 30000, hi: int = 250000, seed: int = 3):
    """Uneven-length EEG-shaped channels (lengths U[lo, hi], alpha U(8, 12) Hz)."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, size=channels)
    alphas = rng.uniform(8.0, 12.0, size=channels)
    return [eeg_like(int(L), seed=1000 + i, alpha_hz=float(a))
            for i, (L, a) in enumerate(zip(lens, alphas))]


def ragged_groups(lengths, groups: int = 8):
    """Channels dealt into `groups` groups of nearly equal total length: longest first, in
    snake order (0..g-1, g-1..0, ...); each group's channel indices in ascending order."""
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    out = [[] for _ in range(groups)]
    for k, i in enumerate(order):
        r, j = divmod(k, groups)
        out[j if r % 2 == 0 else groups - 1 - j].append(i)
    return [sorted(g) for g in out]
