"""ceemdan_gpu_b200 — host-side interface of the B200 ICEEMDAN engine.

The engine is libceemdan_b200.so (CUDA C++ for sm_100a, C ABI in include/ceemdan_b200.h).
This module binds that ABI with ctypes and mirrors the reference entry point

    double iceemdanD(size_t numNoise, size_t SignalLength, size_t num_IMFs, size_t max_iter,
                     int* d_x, double* d_y, double* d_IMFs, double noiseStrength)

(cudaICEEMDAN.cuh:26 of EEGLab-Pannon/CEEMDAN-GPU): same argument names, order and meaning,
device pointers in, [num_IMFs x N] device output.  PyTorch is used only to hold device memory
and to name the current CUDA stream.  There is no CPU fallback: every call raises if the
library is missing or the GPU call fails.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libceemdan_b200.so")

_lib = None


class CeemdanError(RuntimeError):
    """Raised when the engine returns a non-OK ceemdan_status."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(what)


STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "d_x is not the sample index 0..N-1",
    3: "CUDA error",
    4: "out of device memory",
    5: "bounded in-kernel wait ran out",
    6: "cancelled",
}


class Options(ctypes.Structure):
    """ceemdan_options (include/ceemdan_b200.h)."""

    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("noise_sift_cap", ctypes.c_int32),
        ("sd", ctypes.c_double),
        ("sd2", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("d_noise", ctypes.c_void_p),
        ("d_noise_modes_out", ctypes.c_void_p),
        ("h_iters_out", ctypes.POINTER(ctypes.c_int32)),
        ("h_cancel", ctypes.POINTER(ctypes.c_int32)),
        ("group", ctypes.c_int32),
        ("spin_limit", ctypes.c_int32),
        ("h_kernel_ms", ctypes.POINTER(ctypes.c_double)),
        ("h_counters", ctypes.POINTER(ctypes.c_uint64)),
        ("d_noise_state_out", ctypes.c_void_p),
        ("d_noise_state_in", ctypes.c_void_p),
    ]


KERNEL_KINDS = ["extrema", "boundary", "chunk_reduce", "reduced_solve", "segments", "eval",
                "criterion", "sift_small"]
COUNTERS = ["knots", "iterations", "launches", "waves", "peak_bytes"]


def build(force: bool = False) -> str:
    """Compile libceemdan_b200.so for sm_100a with nvcc (ceemdan-gpu_b200/Makefile)."""
    args = ["make", "-C", _HERE]
    if force:
        args.append("-B")
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


_SIZE = ctypes.c_size_t
_VP = ctypes.c_void_p

_ALL_FINISHED = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int)
_EXCHANGE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)


class Split(ctypes.Structure):
    """ceemdan_split (include/ceemdan_b200.h)."""

    _fields_ = [
        ("nr_total", ctypes.c_size_t),
        ("first", ctypes.c_size_t),
        ("rank", ctypes.c_int),
        ("world", ctypes.c_int),
        ("ctx", ctypes.c_void_p),
        ("all_finished", _ALL_FINISHED),
        ("recv_partial", _EXCHANGE),
        ("send_partial", _EXCHANGE),
        ("broadcast_last", _EXCHANGE),
    ]


EXPORTS = {
    # name: (restype, argtypes)
    "ceemdan_default_options": (None, [ctypes.POINTER(Options)]),
    "ceemdan_plain_f64": (ctypes.c_int, [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP, _VP,
                                         ctypes.c_double, ctypes.POINTER(Options), _VP]),
    "ceemdan_plain_f32": (ctypes.c_int, [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP, _VP,
                                         ctypes.c_float, ctypes.POINTER(Options), _VP]),
    "ceemdan_plain_split_f64": (ctypes.c_int, [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP, _VP,
                                               ctypes.c_double, ctypes.POINTER(Options),
                                               ctypes.POINTER(Split), _VP]),
    "ceemdan_batch_f64": (ctypes.c_int, [_SIZE, _VP, _VP, _VP, _SIZE, _SIZE, _SIZE,
                                         ctypes.c_double, ctypes.POINTER(Options), ctypes.c_int]),
    "ceemdan_batched_f64": (ctypes.c_int, [_SIZE, _VP, _VP, _VP, _SIZE, _SIZE, _SIZE,
                                           ctypes.c_double, ctypes.POINTER(Options), _SIZE,
                                           _VP]),
    "ceemdan_noise_cache": (ctypes.c_size_t, [ctypes.c_size_t]),
    "ceemdan_memory_stats": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]),
    "ceemdan_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "ceemdan_last_error": (ctypes.c_char_p, []),
    "ceemdan_build_info": (ctypes.c_char_p, []),
    "ceemdan_kernel_launches": (ctypes.c_uint64, []),
    "ceemdan_envelopes_f64": (ctypes.c_int, [_SIZE, _SIZE, _VP, _VP, _VP, _VP, _VP]),
    "ceemdan_extrema_f64": (ctypes.c_int, [_SIZE, _SIZE, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "ceemdan_tridiag_f64": (ctypes.c_int, [_SIZE, _SIZE, _VP, _VP, _VP, _VP, _VP, _VP]),
    "ceemdan_tridiag_noalloc_f64": (ctypes.c_int, [_SIZE, _SIZE, _VP, _VP, _VP, _VP, _VP, _VP]),
    "ceemdan_canonical_sums_f64": (ctypes.c_int, [_SIZE, _SIZE, _VP, _VP, _VP, _VP, _VP]),
    "ceemdan_forward_taped_f64": (ctypes.c_int, [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP, _VP,
                                                 ctypes.c_double, ctypes.POINTER(Options), _VP,
                                                 ctypes.POINTER(_VP)]),
    "ceemdan_forward_checkpointed_f64": (ctypes.c_int, [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP,
                                                        _VP, ctypes.c_double,
                                                        ctypes.POINTER(Options), _VP,
                                                        ctypes.POINTER(_VP)]),
    "ceemdan_backward_f64": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "ceemdan_tape_bytes": (ctypes.c_size_t, [_VP]),
    "ceemdan_tape_iterations": (ctypes.c_int, [_VP, _SIZE]),
    "ceemdan_tape_free": (None, [_VP]),
}

# C++-linkage drop-in symbols (cudaICEEMDAN.cuh:25-26): double iceemdanS(size_t x4, int*,
# float*, float*, float) and double iceemdanD(size_t x4, int*, double*, double*, double)
DROPIN_SYMBOLS = {"iceemdanS": "_Z9iceemdanSmmmmPiPfS0_f",
                  "iceemdanD": "_Z9iceemdanDmmmmPiPdS0_d"}


def lib():
    """Load libceemdan_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CeemdanError(3, f"{LIB_PATH} is missing: build it with "
                                  "__graft_entry__.build() or `make -C ceemdan-gpu_b200`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        f = getattr(L, DROPIN_SYMBOLS["iceemdanD"])
        f.restype = ctypes.c_double
        f.argtypes = [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP, _VP, ctypes.c_double]
        f = getattr(L, DROPIN_SYMBOLS["iceemdanS"])
        f.restype = ctypes.c_double
        f.argtypes = [_SIZE, _SIZE, _SIZE, _SIZE, _VP, _VP, _VP, ctypes.c_float]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        detail = lib().ceemdan_last_error().decode(errors="replace")
        raise CeemdanError(rc, f"{STATUS.get(rc, 'error')} ({detail})")


def _require(ok, what: str):
    """Argument check of the Python entry points: CeemdanError with status 1 (invalid
    argument), raised before anything is launched."""
    if not ok:
        raise CeemdanError(1, f"invalid argument ({what})")


def default_options() -> Options:
    o = Options()
    lib().ceemdan_default_options(ctypes.byref(o))
    return o


def _stream_handle(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


# ---------------------------------------------------------------------------------------
# reference-shaped entry point
# ---------------------------------------------------------------------------------------
def iceemdanD(numNoise: int, SignalLength: int, num_IMFs: int, max_iter: int, d_x: int,
              d_y: int, d_IMFs: int, noiseStrength: float) -> float:
    """The reference's iceemdanD: raw device pointers in (ints), seconds of the CEEMDAN
    stages out.  Noise: cuRAND XORWOW seed 1234 (cudaICEEMDAN.cu:1460-1462).  Raises
    CeemdanError where the reference would silently produce garbage."""
    f = getattr(lib(), DROPIN_SYMBOLS["iceemdanD"])
    t = f(numNoise, SignalLength, num_IMFs, max_iter, d_x, d_y, d_IMFs, noiseStrength)
    if t < 0:
        _check(int(round(-t)))
    return t


def iceemdanS(numNoise: int, SignalLength: int, num_IMFs: int, max_iter: int, d_x: int,
              d_y: int, d_IMFs: int, noiseStrength: float) -> float:
    """The reference's iceemdanS (float data): raw device pointers in (ints), seconds of the
    CEEMDAN stages out.  Noise: cuRAND XORWOW seed 1234 float normals (cudaICEEMDAN.cu:741).
    Computes in FP64 on the exactly widened data; IMFs rounded to float."""
    f = getattr(lib(), DROPIN_SYMBOLS["iceemdanS"])
    t = f(numNoise, SignalLength, num_IMFs, max_iter, d_x, d_y, d_IMFs, noiseStrength)
    if t < 0:
        _check(int(round(-t)))
    return t


# ---------------------------------------------------------------------------------------
# tensor-level helpers (torch CUDA tensors)
# ---------------------------------------------------------------------------------------
def iceemdan(y, numNoise: int, num_IMFs: int, max_iter: int, noiseStrength: float, *,
             noise=None, seed: int = 1234, noise_sift_cap: int = 2000, sd: float = 0.05,
             sd2: float = 0.5, tol: float = 0.05, return_iters: bool = False,
             return_noise_modes: bool = False, group: int = 0, profile: dict | None = None,
             x=None, stream=None, noise_state=None, return_noise_state: bool = False,
             cancel=None, spin_limit: int = 0):
    """ICEEMDAN of one CUDA tensor y [N] -> IMFs [num_IMFs, N] (CUDA, y's dtype).

    float64 y runs ceemdan_plain_f64 (iceemdanD); float32 y runs ceemdan_plain_f32 (iceemdanS:
    FP64 computation on the widened data, default noise from cuRAND's float normals, IMFs
    rounded to float).  noise: optional [numNoise, N] float64 CUDA tensor of N(0,1)
    realizations; default is cuRAND XORWOW with `seed`, as the reference generates it.  profile: optional dict that
    receives per-kernel device milliseconds ("ms") and work counters ("counters").  x:
    optional int32 CUDA tensor of sample coordinates (d_x of the reference; must be 0..N-1,
    built here when omitted).  return_noise_state: also return the state the noise phase
    leaves (float64 [(num_IMFs+1)*numNoise*N + numNoise]); noise_state: start from such a state
    and skip the noise phase -- for channels of the same length and noise this gives the
    full call's result bit for bit.  cancel: optional ctypes.c_int32 host word; nonzero stops
    the call between groups of sift iterations (CeemdanError with status 6).  spin_limit: polls
    of the on-chip path's stop test before it gives up (status 5); see ceemdan_options."""
    import torch
    _require(y.is_cuda and y.dtype in (torch.float64, torch.float32) and y.dim() == 1,
             "y must be a 1-D float64 or float32 CUDA tensor")
    y = y.contiguous()
    n = y.numel()
    if x is None:
        x = torch.arange(n, dtype=torch.int32, device=y.device)
    _require(x.is_cuda and x.dtype == torch.int32 and x.numel() == n,
             "x must be an int32 CUDA tensor of N sample coordinates")
    imfs = torch.empty((num_IMFs, n), dtype=y.dtype, device=y.device)
    o = default_options()
    o.noise_sift_cap = noise_sift_cap
    o.sd, o.sd2, o.tol = sd, sd2, tol
    o.seed = seed
    o.group = group
    o.spin_limit = spin_limit
    if cancel is not None:
        o.h_cancel = ctypes.pointer(cancel)
    if noise is not None:
        _require(noise.is_cuda and noise.dtype == torch.float64 and noise.shape == (numNoise, n),
                 "noise must be a float64 CUDA tensor of shape [numNoise, N]")
        noise = noise.contiguous()
        o.d_noise = noise.data_ptr()
    iters = (ctypes.c_int32 * (2 * (num_IMFs - 1)))()
    o.h_iters_out = ctypes.cast(iters, ctypes.POINTER(ctypes.c_int32))
    kms = (ctypes.c_double * len(KERNEL_KINDS))()
    ctr = (ctypes.c_uint64 * len(COUNTERS))()
    if profile is not None:
        o.h_kernel_ms = ctypes.cast(kms, ctypes.POINTER(ctypes.c_double))
        o.h_counters = ctypes.cast(ctr, ctypes.POINTER(ctypes.c_uint64))
    state = None
    if return_noise_state:
        state = torch.empty(((num_IMFs + 1) * numNoise * n + numNoise,), dtype=torch.float64,
                            device=y.device)
        o.d_noise_state_out = state.data_ptr()
    if noise_state is not None:
        _require(noise_state.is_cuda and noise_state.dtype == torch.float64
                 and noise_state.numel() == (num_IMFs + 1) * numNoise * n + numNoise,
                 "noise_state must be a float64 CUDA tensor of "
                 "(num_IMFs+1)*numNoise*N + numNoise values")
        noise_state = noise_state.contiguous()
        o.d_noise_state_in = noise_state.data_ptr()
    modes = None
    if return_noise_modes:
        modes = torch.empty((num_IMFs, numNoise, n), dtype=torch.float64, device=y.device)
        o.d_noise_modes_out = modes.data_ptr()
    plain = lib().ceemdan_plain_f64 if y.dtype == torch.float64 else lib().ceemdan_plain_f32
    rc = plain(numNoise, n, num_IMFs, max_iter, _ptr(x), _ptr(y), _ptr(imfs), noiseStrength,
               ctypes.byref(o), _stream_handle(stream))
    _check(rc)
    if profile is not None:
        profile["ms"] = dict(zip(KERNEL_KINDS, list(kms)))
        profile["counters"] = dict(zip(COUNTERS, [int(v) for v in ctr]))
    out = [imfs]
    if return_iters:
        out.append(list(iters))
    if return_noise_modes:
        out.append(modes)
    if return_noise_state:
        out.append(state)
    return out[0] if len(out) == 1 else tuple(out)


def memory_stats(reset_peak: bool = False) -> dict:
    """The library's device memory pool on the current device: bytes in use by calls, their
    high-water mark, bytes reserved (ceemdan_memory_stats)."""
    u, p, r = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().ceemdan_memory_stats(ctypes.byref(u), ctypes.byref(p), ctypes.byref(r),
                                      1 if reset_peak else 0))
    return {"used": u.value, "peak": p.value, "reserved": r.value}


def envelopes(h, stream=None):
    """Upper/lower spline envelopes of every row of h [nr, N] (float64 CUDA) and the knot
    counts [2, nr] (maxima, minima)."""
    import torch
    h = h.contiguous()
    nr, n = h.shape
    up = torch.empty_like(h)
    lo = torch.empty_like(h)
    cnt = torch.empty((2, nr), dtype=torch.int32, device=h.device)
    _check(lib().ceemdan_envelopes_f64(nr, n, _ptr(h), _ptr(up), _ptr(lo), _ptr(cnt),
                                       _stream_handle(stream)))
    return up, lo, cnt


def extrema(h, stream=None):
    """Knots of every row of h [nr, N]: (kx_max, ky_max, kx_min, ky_min, counts[2, nr]);
    row r's knots occupy the first counts[., r] entries of row r."""
    import torch
    h = h.contiguous()
    nr, n = h.shape
    kxM = torch.zeros((nr, n), dtype=torch.int32, device=h.device)
    kyM = torch.zeros((nr, n), dtype=torch.float64, device=h.device)
    kxm = torch.zeros_like(kxM)
    kym = torch.zeros_like(kyM)
    cnt = torch.empty((2, nr), dtype=torch.int32, device=h.device)
    _check(lib().ceemdan_extrema_f64(nr, n, _ptr(h), _ptr(kxM), _ptr(kyM), _ptr(kxm), _ptr(kym),
                                     _ptr(cnt), _stream_handle(stream)))
    return kxM, kyM, kxm, kym, cnt


def tridiag(l, m, u, r, stream=None):
    """Canonical partitioned solve of batch x n tridiagonal systems (float64 CUDA)."""
    import torch
    l, m, u, r = (t.contiguous() for t in (l, m, u, r))
    batch, n = l.shape
    x = torch.empty_like(r)
    _check(lib().ceemdan_tridiag_f64(batch, n, _ptr(l), _ptr(m), _ptr(u), _ptr(r), _ptr(x),
                                     _stream_handle(stream)))
    return x


def tridiag_noalloc(l, m, u, r, x, stream=None):
    """ceemdan_tridiag_noalloc_f64: the canonical solve into the caller's x, using only the
    library's static device scratch (no allocation by the library; the caller provides
    every input and output buffer).  Limit: batch*(5*n+64) <= 1048576 doubles."""
    batch, n = l.shape
    _check(lib().ceemdan_tridiag_noalloc_f64(batch, n, _ptr(l), _ptr(m), _ptr(u), _ptr(r),
                                             _ptr(x), _stream_handle(stream)))
    return x


def canonical_sums(v, mean=None, stream=None):
    """Canonical sums (and squared deviations from mean) of the rows of v [batch, n]."""
    import torch
    v = v.contiguous()
    batch, n = v.shape
    s = torch.empty(batch, dtype=torch.float64, device=v.device)
    q = torch.empty(batch, dtype=torch.float64, device=v.device) if mean is not None else None
    mp = _ptr(mean.contiguous()) if mean is not None else None
    _check(lib().ceemdan_canonical_sums_f64(batch, n, _ptr(v), mp, _ptr(s),
                                            _ptr(q) if q is not None else None,
                                            _stream_handle(stream)))
    return (s, q) if mean is not None else s


def iceemdan_batch(channels, numNoise: int, num_IMFs: int, max_iter: int, noiseStrength: float,
                   *, seed: int = 1234, streams: int = 4, noise_sift_cap: int = 2000,
                   sd: float = 0.05, sd2: float = 0.5, tol: float = 0.05):
    """ceemdan_batch_f64 on a list of float64 CUDA tensors of different lengths: the IMFs of
    each (list of [num_IMFs, N_c] tensors); channel c uses cuRAND seed `seed + c`."""
    import torch
    ys = [y.contiguous() for y in channels]
    for y in ys:
        _require(y.is_cuda and y.dtype == torch.float64 and y.dim() == 1,
                 "every channel must be a 1-D float64 CUDA tensor")
    outs = [torch.empty((num_IMFs, y.numel()), dtype=torch.float64, device=y.device) for y in ys]
    torch.cuda.synchronize()
    k = len(ys)
    lengths = (ctypes.c_size_t * k)(*[y.numel() for y in ys])
    yp = (ctypes.c_void_p * k)(*[y.data_ptr() for y in ys])
    op = (ctypes.c_void_p * k)(*[o.data_ptr() for o in outs])
    o = default_options()
    o.noise_sift_cap = noise_sift_cap
    o.sd, o.sd2, o.tol = sd, sd2, tol
    o.seed = seed
    _check(lib().ceemdan_batch_f64(k, lengths, yp, op, numNoise, num_IMFs, max_iter,
                                   noiseStrength, ctypes.byref(o), streams))
    return outs


def iceemdan_batched(channels, numNoise: int, num_IMFs: int, max_iter: int,
                     noiseStrength: float, *, seed: int = 1234, noise_sift_cap: int = 2000,
                     sd: float = 0.05, sd2: float = 0.5, tol: float = 0.05, group: int = 0,
                     wave_bytes: int = 0, return_iters: bool = False,
                     profile: dict | None = None, stream=None, cancel=None):
    """ceemdan_batched_f64 on a list of float64 CUDA tensors of different lengths: the IMFs of
    each channel (list of [num_IMFs, N_c] tensors), each equal bit for bit to iceemdan() of
    that channel with cuRAND seed `seed + c`.  All channels of a wave sift together in one
    device-driven loop (CUDA graph); waves of at most wave_bytes (0 = 85% of the free device
    memory).  return_iters: also return [channels][2*(num_IMFs-1)] iteration counts (noise
    stages, then CEEMDAN stages).  profile: optional dict that receives per-kernel device
    milliseconds ("ms") and counters ("counters": knots, loop iterations, launches, waves,
    peak pool bytes)."""
    import torch
    ys = [y.contiguous() for y in channels]
    for y in ys:
        _require(y.is_cuda and y.dtype == torch.float64 and y.dim() == 1,
                 "every channel must be a 1-D float64 CUDA tensor")
    outs = [torch.empty((num_IMFs, y.numel()), dtype=torch.float64, device=y.device)
            for y in ys]
    k = len(ys)
    lengths = (ctypes.c_size_t * k)(*[y.numel() for y in ys])
    yp = (ctypes.c_void_p * k)(*[y.data_ptr() for y in ys])
    op = (ctypes.c_void_p * k)(*[o.data_ptr() for o in outs])
    o = default_options()
    o.noise_sift_cap = noise_sift_cap
    o.sd, o.sd2, o.tol = sd, sd2, tol
    o.seed = seed
    o.group = group
    if cancel is not None:
        o.h_cancel = ctypes.pointer(cancel)
    iters = (ctypes.c_int32 * (k * 2 * (num_IMFs - 1)))()
    if return_iters:
        o.h_iters_out = ctypes.cast(iters, ctypes.POINTER(ctypes.c_int32))
    kms = (ctypes.c_double * len(KERNEL_KINDS))()
    ctr = (ctypes.c_uint64 * len(COUNTERS))()
    if profile is not None:
        o.h_kernel_ms = ctypes.cast(kms, ctypes.POINTER(ctypes.c_double))
        o.h_counters = ctypes.cast(ctr, ctypes.POINTER(ctypes.c_uint64))
    _check(lib().ceemdan_batched_f64(k, lengths, yp, op, numNoise, num_IMFs, max_iter,
                                     noiseStrength, ctypes.byref(o), wave_bytes,
                                     _stream_handle(stream)))
    if profile is not None:
        profile["ms"] = dict(zip(KERNEL_KINDS, list(kms)))
        profile["counters"] = dict(zip(COUNTERS, [int(v) for v in ctr]))
    if return_iters:
        m = 2 * (num_IMFs - 1)
        it = list(iters)
        return outs, [it[c * m:(c + 1) * m] for c in range(k)]
    return outs


# ---------------------------------------------------------------------------------------
# reverse pass: taped forward, vector-Jacobian product, torch.autograd binding
# ---------------------------------------------------------------------------------------
class Tape:
    """Frozen structure of one taped forward call (ceemdan_forward_taped_f64): knot positions,
    end-rule choices, marks and iteration counts of every signal-stage sift, the noise modes
    and the stage statistics.  backward(g) returns (d imfs / d y)^T g for that structure."""

    def __init__(self, handle, num_imfs: int, n: int, device):
        self._h = handle
        self.num_imfs = num_imfs
        self.n = n
        self.device = device

    @property
    def bytes(self) -> int:
        return int(lib().ceemdan_tape_bytes(self._h)) if self._h else 0

    @property
    def iterations(self):
        """Executed lock-step iterations of each signal stage."""
        return [int(lib().ceemdan_tape_iterations(self._h, i)) for i in range(self.num_imfs - 1)]

    def backward(self, grad_imfs, stream=None):
        """grad_y [N] (float64 CUDA) = (d imfs / d y)^T grad_imfs [num_IMFs, N]."""
        import torch
        if not self._h:
            raise CeemdanError(1, "the tape has been freed")
        g = grad_imfs.to(device=self.device, dtype=torch.float64).contiguous()
        _require(g.shape == (self.num_imfs, self.n), "grad_imfs must have shape [num_IMFs, N]")
        gy = torch.empty(self.n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _check(lib().ceemdan_backward_f64(self._h, _ptr(g), _ptr(gy), _stream_handle(stream)))
        return gy

    def free(self):
        if self._h:
            lib().ceemdan_tape_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class _DeviceDoubles:
    """A zero-copy view of n doubles at a device address (CUDA array interface), for
    torch.as_tensor."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 2}


def iceemdan_split(y, nr_total: int, first: int, nr_local: int, num_IMFs: int, max_iter: int,
                   noiseStrength: float, ensemble, *, noise=None, seed: int = 1234,
                   noise_sift_cap: int = 2000, sd: float = 0.05, sd2: float = 0.5,
                   tol: float = 0.05, x=None, stream=None, return_iters: bool = False):
    """One part of a channel whose realizations are split over the ranks of a process group
    (ceemdan_plain_split_f64): this rank holds realizations first .. first + nr_local - 1 of
    nr_total (contiguous blocks in rank order, multichannel.realization_block).  ensemble gives
    the exchanges (multichannel.OrderedEnsemble: all_finished every sift iteration, the
    ordered running sums of every CEEMDAN stage); its tensors live on ensemble.device (CPU
    tensors for gloo, this GPU for NCCL).  noise: this part's [nr_local, N] rows, else cuRAND
    with `seed` over the whole ensemble.  Every rank returns the whole channel's IMFs, bit for
    bit those of iceemdan() with all nr_total realizations."""
    import torch
    _require(y.is_cuda and y.dtype == torch.float64 and y.dim() == 1,
             "y must be a 1-D float64 CUDA tensor")
    y = y.contiguous()
    n = y.numel()
    if x is None:
        x = torch.arange(n, dtype=torch.int32, device=y.device)
    imfs = torch.empty((num_IMFs, n), dtype=torch.float64, device=y.device)
    o = default_options()
    o.noise_sift_cap = noise_sift_cap
    o.sd, o.sd2, o.tol = sd, sd2, tol
    o.seed = seed
    if noise is not None:
        noise = noise.contiguous()
        _require(noise.is_cuda and noise.dtype == torch.float64 and noise.shape == (nr_local, n),
                 "noise must be a float64 CUDA tensor of shape [nr_local, N]")
        o.d_noise = noise.data_ptr()
    iters = (ctypes.c_int32 * (2 * (num_IMFs - 1)))()
    o.h_iters_out = ctypes.cast(iters, ctypes.POINTER(ctypes.c_int32))
    dev = torch.device(getattr(ensemble, "device", None) or "cpu")
    errors = []

    def view(ptr, count):
        return torch.as_tensor(_DeviceDoubles(ptr, count), device=y.device)

    def exchange(fn, ptr, count, write):
        # the engine's stream is idle here; torch's device work completes before returning
        try:
            t = view(ptr, count)
            buf = t if dev.type == "cuda" else t.cpu()
            fn(buf)
            if write and buf is not t:
                t.copy_(buf)
            torch.cuda.synchronize(y.device)
            return 0
        except Exception as e:  # reported after the call returns
            errors.append(e)
            return 1

    def all_finished(_ctx, local):
        try:
            return 1 if ensemble.all_finished(bool(local)) else 0
        except Exception as e:
            errors.append(e)
            return -1

    sp = Split()
    sp.nr_total, sp.first = nr_total, first
    sp.rank, sp.world = ensemble.rank, ensemble.world
    sp.all_finished = _ALL_FINISHED(all_finished)
    sp.recv_partial = _EXCHANGE(lambda c, p, k: exchange(ensemble.recv_partial, p, k, True))
    sp.send_partial = _EXCHANGE(lambda c, p, k: exchange(ensemble.send_partial, p, k, False))
    sp.broadcast_last = _EXCHANGE(lambda c, p, k: exchange(ensemble.broadcast_last, p, k, True))
    rc = lib().ceemdan_plain_split_f64(nr_local, n, num_IMFs, max_iter, _ptr(x), _ptr(y),
                                       _ptr(imfs), noiseStrength, ctypes.byref(o),
                                       ctypes.byref(sp), _stream_handle(stream))
    if errors:
        raise errors[0]
    _check(rc)
    if return_iters:
        return imfs, list(iters)
    return imfs


def iceemdan_taped(y, numNoise: int, num_IMFs: int, max_iter: int, noiseStrength: float, *,
                   noise=None, seed: int = 1234, noise_sift_cap: int = 2000, sd: float = 0.05,
                   sd2: float = 0.5, tol: float = 0.05, x=None, stream=None, noise_state=None,
                   checkpoint: bool = False, counters: dict | None = None):
    """iceemdan() of a float64 CUDA tensor that also records the tape of its reverse pass:
    returns (imfs [num_IMFs, N], Tape).  The IMFs equal iceemdan()'s bit for bit.
    noise_state: a state from iceemdan(..., return_noise_state=True) for the same length,
    noise and options (skips the noise phase, same result).  checkpoint: keep per-stage
    checkpoints instead of every iteration (ceemdan_forward_checkpointed_f64; the backward
    re-runs each stage, same gradients, memory independent of the iteration counts).
    counters: optional dict that receives the forward's work counters (no kernel timing)."""
    import torch
    _require(y.is_cuda and y.dtype == torch.float64 and y.dim() == 1,
             "y must be a 1-D float64 CUDA tensor")
    y = y.contiguous()
    n = y.numel()
    if x is None:
        x = torch.arange(n, dtype=torch.int32, device=y.device)
    imfs = torch.empty((num_IMFs, n), dtype=torch.float64, device=y.device)
    o = default_options()
    o.noise_sift_cap = noise_sift_cap
    o.sd, o.sd2, o.tol = sd, sd2, tol
    o.seed = seed
    if noise is not None:
        _require(noise.is_cuda and noise.dtype == torch.float64 and noise.shape == (numNoise, n),
                 "noise must be a float64 CUDA tensor of shape [numNoise, N]")
        noise = noise.contiguous()
        o.d_noise = noise.data_ptr()
    if noise_state is not None:
        _require(noise_state.is_cuda and noise_state.dtype == torch.float64
                 and noise_state.numel() == (num_IMFs + 1) * numNoise * n + numNoise,
                 "noise_state must be a float64 CUDA tensor of "
                 "(num_IMFs+1)*numNoise*N + numNoise values")
        noise_state = noise_state.contiguous()
        o.d_noise_state_in = noise_state.data_ptr()
    ctr = (ctypes.c_uint64 * len(COUNTERS))()
    if counters is not None:
        o.h_counters = ctypes.cast(ctr, ctypes.POINTER(ctypes.c_uint64))
    h = _VP()
    with torch.cuda.device(y.device):
        fwd = (lib().ceemdan_forward_checkpointed_f64 if checkpoint
               else lib().ceemdan_forward_taped_f64)
        _check(fwd(numNoise, n, num_IMFs, max_iter, _ptr(x), _ptr(y), _ptr(imfs), noiseStrength,
                   ctypes.byref(o), _stream_handle(stream), ctypes.byref(h)))
    if counters is not None:
        counters.update(zip(COUNTERS, [int(v) for v in ctr]))
    return imfs, Tape(h, num_IMFs, n, y.device)


_autograd_fn = None


def _function():
    global _autograd_fn
    if _autograd_fn is None:
        import torch

        class ICEEMDANFunction(torch.autograd.Function):
            """imfs = ICEEMDAN(y); backward: ceemdan_backward_f64 on the forward's tape."""

            @staticmethod
            def forward(ctx, y, numNoise, num_IMFs, max_iter, noiseStrength, noise, seed,
                        noise_sift_cap):
                imfs, tape = iceemdan_taped(y.detach(), numNoise, num_IMFs, max_iter,
                                            noiseStrength, noise=noise, seed=seed,
                                            noise_sift_cap=noise_sift_cap)
                ctx.tape = tape
                return imfs

            @staticmethod
            def backward(ctx, grad_imfs):
                gy = ctx.tape.backward(grad_imfs)
                ctx.tape.free()
                return gy, None, None, None, None, None, None, None

        _autograd_fn = ICEEMDANFunction
    return _autograd_fn


def iceemdan_autograd(y, numNoise: int, num_IMFs: int, max_iter: int, noiseStrength: float, *,
                      noise=None, seed: int = 1234, noise_sift_cap: int = 2000):
    """Differentiable ICEEMDAN of a float64 CUDA tensor (torch.autograd): the forward is the
    taped decomposition, the backward its reverse pass with the forward's structure (knots,
    end rules, stop decisions) frozen.  A second backward through the same graph is not
    supported (the tape is freed after the first)."""
    return _function().apply(y, numNoise, num_IMFs, max_iter, noiseStrength, noise, seed,
                             noise_sift_cap)
