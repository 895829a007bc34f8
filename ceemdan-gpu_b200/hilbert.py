"""Hilbert spectral analysis of IMFs: the time-frequency step that follows the decomposition.

The reference stops at the IMFs; its stated use is EEG time-frequency analysis (the
Hilbert-Huang transform: instantaneous amplitude and frequency of every IMF).  This module
computes, for IMFs [K, N] (torch tensors on the GPU or the CPU, float64 or float32):

  analytic(imfs)            z = x + i H(x), the analytic signal of each row, by the FFT
                            definition (scipy.signal.hilbert): Z = F(x) * h with h = 1 at DC
                            (and at Nyquist for even N), 2 for the positive frequencies, 0
                            for the negative ones; z = F^-1(Z).
  amplitude(imfs)           |z|
  phase(imfs)               unwrapped angle of z (radians)
  inst_frequency(imfs, fs)  d(phase)/dt / (2 pi), first differences: [K, N-1] in Hz

The FFTs run through torch.fft (cuFFT on CUDA tensors); this step is outside the
decomposition's hot path.
"""
from __future__ import annotations

import math


def _torch():
    import torch
    return torch


def analytic(imfs):
    """Analytic signal of each row of imfs ([K, N] or [N]); complex128 for float64 input,
    complex64 for float32."""
    torch = _torch()
    x = imfs if imfs.dim() == 2 else imfs.unsqueeze(0)
    n = x.shape[-1]
    if n < 1:
        raise ValueError("empty signal")
    spec = torch.fft.fft(x, dim=-1)
    h = torch.zeros(n, dtype=x.dtype, device=x.device)
    h[0] = 1.0
    if n % 2 == 0:
        h[n // 2] = 1.0
        h[1:n // 2] = 2.0
    else:
        h[1:(n + 1) // 2] = 2.0
    z = torch.fft.ifft(spec * h, dim=-1)
    return z if imfs.dim() == 2 else z[0]


def amplitude(imfs):
    """Instantaneous amplitude |z| of each row."""
    return analytic(imfs).abs()


def phase(imfs):
    """Unwrapped instantaneous phase of each row (radians, numpy.unwrap semantics)."""
    torch = _torch()
    ang = torch.angle(analytic(imfs))
    d = torch.diff(ang, dim=-1)
    # wrap the increments into [-pi, pi), keeping +pi for positive jumps (numpy.unwrap)
    dm = torch.remainder(d + math.pi, 2 * math.pi) - math.pi
    dm = torch.where((dm == -math.pi) & (d > 0), torch.full_like(dm, math.pi), dm)
    corr = torch.where(d.abs() < math.pi, torch.zeros_like(d), dm - d)
    out = ang.clone()
    out[..., 1:] += torch.cumsum(corr, dim=-1)
    return out


def inst_frequency(imfs, fs: float):
    """Instantaneous frequency (Hz) from first differences of the unwrapped phase:
    [K, N-1] (or [N-1])."""
    torch = _torch()
    return torch.diff(phase(imfs), dim=-1) * (fs / (2 * math.pi))
