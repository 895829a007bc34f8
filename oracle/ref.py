"""ctypes binding of oracle/_ref/libref_iceemdan.so: the reference's own CUDA implementation
built from its sources by oracle/build_ref.sh (test infrastructure only; needs a GPU).

Full iceemdanD runs use only configurations without partially-exited warps in the
reference's barrier code: N a multiple of 256 (meanD/varianceD return before their block
reduction when tid >= N) and NR a multiple of 32 (checkBreak synchronises inside
`if (noiseIdx < numNoise)`).  The envelope pass has no block barriers.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(_HERE, "_ref", "libref_iceemdan.so")
_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def available() -> bool:
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(SO)
        L.ref_iceemdan_f64.argtypes = [ctypes.c_size_t] * 4 + [_dp, _dp, ctypes.c_double, _dp]
        L.ref_iceemdan_f64.restype = ctypes.c_int
        L.ref_envelopes_f64.argtypes = [ctypes.c_size_t, ctypes.c_size_t, _dp, _dp, _dp, _ip]
        L.ref_envelopes_f64.restype = ctypes.c_int
        L.ref_knots_f64.argtypes = [ctypes.c_size_t, ctypes.c_size_t, _dp, _ip, _dp, _ip, _dp,
                                    _ip]
        L.ref_knots_f64.restype = ctypes.c_int
        _lib = L
    return _lib


def _check_shape(nr, n):
    if n % 256 or nr % 32:
        raise ValueError("reference runs need N % 256 == 0 and NR % 32 == 0")


def iceemdan(y, nr, num_imfs, max_iter, nstd):
    """iceemdanD of the reference (cuRAND XORWOW seed 1234 noise inside).  Returns the IMFs
    [num_imfs, n] and the seconds the reference reports."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = y.size
    _check_shape(nr, n)
    imfs = np.zeros((num_imfs, n))
    secs = ctypes.c_double()
    rc = lib().ref_iceemdan_f64(nr, n, num_imfs, max_iter, y.ctypes.data_as(_dp),
                                imfs.ctypes.data_as(_dp), nstd, ctypes.byref(secs))
    if rc:
        raise RuntimeError(f"reference iceemdanD: CUDA error {rc}")
    return imfs, secs.value


def envelopes(h):
    """Upper/lower envelopes of every row of h [nr, n] from the reference's kernels, and the
    knot counts [2, nr]."""
    h = np.ascontiguousarray(h, dtype=np.float64)
    nr, n = h.shape
    up = np.zeros_like(h)
    lo = np.zeros_like(h)
    cnt = np.zeros((2, nr), dtype=np.int32)
    rc = lib().ref_envelopes_f64(nr, n, h.ctypes.data_as(_dp), up.ctypes.data_as(_dp),
                                 lo.ctypes.data_as(_dp), cnt.ctypes.data_as(_ip))
    if rc:
        raise RuntimeError(f"reference envelopes: CUDA error {rc}")
    return up, lo, cnt


def knots(h):
    """Knots of every row of h [nr, n] from the reference's extrema, scan, compaction and
    end-knot kernels: (kx_max, ky_max, kx_min, ky_min) as [nr, n] arrays (row r's knots in
    its first counts[., r] entries) and counts [2, nr]."""
    h = np.ascontiguousarray(h, dtype=np.float64)
    nr, n = h.shape
    kxM = np.zeros((nr, n), dtype=np.int32)
    kyM = np.zeros((nr, n))
    kxm = np.zeros((nr, n), dtype=np.int32)
    kym = np.zeros((nr, n))
    cnt = np.zeros((2, nr), dtype=np.int32)
    rc = lib().ref_knots_f64(nr, n, h.ctypes.data_as(_dp), kxM.ctypes.data_as(_ip),
                             kyM.ctypes.data_as(_dp), kxm.ctypes.data_as(_ip),
                             kym.ctypes.data_as(_dp), cnt.ctypes.data_as(_ip))
    if rc:
        raise RuntimeError(f"reference knots: CUDA error {rc}")
    return kxM, kyM, kxm, kym, cnt
