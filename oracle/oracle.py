"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module,
and only as the checker or the timed CPU baseline.  It wraps liboracle_ceemdan.so, the
C++/OpenMP restatement of iceemdanD (cudaICEEMDAN.cu:1340-2059) built by oracle/Makefile.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle_ceemdan.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class OracleOpts(ctypes.Structure):
    _fields_ = [
        ("noise_sift_cap", ctypes.c_int),
        ("sd", ctypes.c_double),
        ("sd2", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("solver", ctypes.c_int),
        ("chunk", ctypes.c_int),
        ("threads", ctypes.c_int),
        ("iters_out", _ip),
        ("noise_modes_out", _dp),
    ]


def build(force: bool = False) -> str:
    """Compile liboracle_ceemdan.so with oracle/Makefile (g++, OpenMP)."""
    if force or not os.path.exists(_SO):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "-s"], check=True,
                       stdout=subprocess.DEVNULL)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.oracle_default_opts.argtypes = [ctypes.POINTER(OracleOpts)]
        L.oracle_iceemdan_f64.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                          ctypes.c_size_t, _dp, _dp, ctypes.c_double, _dp,
                                          ctypes.POINTER(OracleOpts)]
        L.oracle_iceemdan_f64.restype = ctypes.c_int
        L.oracle_extrema_f64.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _ip, _dp]
        L.oracle_extrema_f64.restype = ctypes.c_int
        L.oracle_boundary_f64.argtypes = [ctypes.c_int, _ip, _dp, ctypes.c_int]
        L.oracle_spline_solve_f64.argtypes = [ctypes.c_int, _ip, _dp, _dp, ctypes.c_int,
                                              ctypes.c_int]
        L.oracle_spline_eval_f64.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _dp]
        L.oracle_canonical_sum_f64.argtypes = [_dp, ctypes.c_size_t]
        L.oracle_canonical_sum_f64.restype = ctypes.c_double
        L.oracle_canonical_sqdev_f64.argtypes = [_dp, ctypes.c_size_t, ctypes.c_double]
        L.oracle_canonical_sqdev_f64.restype = ctypes.c_double
        L.oracle_tridiag_partitioned_f64.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, _dp,
                                                     ctypes.c_int]
        L.oracle_tape_forward_f64.argtypes = [ctypes.c_size_t, ctypes.c_size_t,
                                              ctypes.c_size_t, ctypes.c_size_t, _dp, _dp,
                                              ctypes.c_double, _dp, ctypes.POINTER(OracleOpts)]
        L.oracle_tape_forward_f64.restype = ctypes.c_void_p
        L.oracle_tape_forward_shared_f64.argtypes = [ctypes.c_size_t, ctypes.c_size_t,
                                                     ctypes.c_size_t, ctypes.c_size_t, _dp,
                                                     ctypes.c_double, _dp,
                                                     ctypes.POINTER(OracleOpts), ctypes.c_void_p]
        L.oracle_tape_forward_shared_f64.restype = ctypes.c_void_p
        L.oracle_tape_replay_f64.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.oracle_tape_vjp_f64.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.oracle_tape_vjp_recompute_f64.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.oracle_tape_recompute_mismatches.argtypes = [ctypes.c_void_p]
        L.oracle_tape_iterations.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_tape_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, _ip,
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.oracle_tape_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def iceemdan(y, noise, num_imfs, max_iter, nstd, *, solver=0, chunk=16, threads=0,
             noise_sift_cap=2000, sd=0.05, sd2=0.5, tol=0.05, return_iters=False,
             return_noise_modes=False):
    """Oracle ICEEMDAN.  y: [n] f64, noise: [nr, n] f64.  Returns imfs [num_imfs, n]
    (and, if asked, the per-stage lock-step iteration counts and the noise modes)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    nr, n = noise.shape
    assert y.shape == (n,)
    imfs = np.zeros((num_imfs, n), dtype=np.float64)
    o = OracleOpts()
    lib().oracle_default_opts(ctypes.byref(o))
    o.noise_sift_cap = noise_sift_cap
    o.sd, o.sd2, o.tol = sd, sd2, tol
    o.solver, o.chunk, o.threads = solver, chunk, threads
    iters = np.zeros(2 * (num_imfs - 1), dtype=np.int32)
    o.iters_out = _i(iters)
    modes = None
    if return_noise_modes:
        modes = np.zeros((num_imfs, nr, n), dtype=np.float64)
        o.noise_modes_out = _d(modes)
    rc = lib().oracle_iceemdan_f64(nr, n, num_imfs, max_iter, _d(y), _d(noise), nstd,
                                   _d(imfs), ctypes.byref(o))
    if rc != 0:
        raise ValueError(f"oracle_iceemdan_f64 rejected its arguments (code {rc})")
    out = [imfs]
    if return_iters:
        out.append(iters)
    if return_noise_modes:
        out.append(modes)
    return out[0] if len(out) == 1 else tuple(out)


class _Split(ctypes.Structure):
    _fields_ = [
        ("nr_total", ctypes.c_size_t),
        ("rank", ctypes.c_int),
        ("world", ctypes.c_int),
        ("ctx", ctypes.c_void_p),
        ("all_finished", ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int)),
        ("recv_partial", ctypes.CFUNCTYPE(None, ctypes.c_void_p, _dp, ctypes.c_size_t)),
        ("send_partial", ctypes.CFUNCTYPE(None, ctypes.c_void_p, _dp, ctypes.c_size_t)),
        ("broadcast_last", ctypes.CFUNCTYPE(None, ctypes.c_void_p, _dp, ctypes.c_size_t)),
    ]


def iceemdan_split(y, noise_local, nr_total, rank, world, ops, num_imfs, max_iter, nstd, *,
                   solver=1, chunk=16, threads=0, noise_sift_cap=2000, return_iters=False):
    """Oracle ICEEMDAN of one part of a realization split (oracle_iceemdan_split_f64):
    noise_local holds this part's contiguous block of realizations; `ops` supplies the
    exchanges -- ops.all_finished(bool) -> bool, ops.recv_partial(t), ops.send_partial(t),
    ops.broadcast_last(t) on float64 numpy arrays of n samples (filled in place when
    receiving).  Returns the whole channel's IMFs (and the iteration counts)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    noise_local = np.ascontiguousarray(noise_local, dtype=np.float64)
    nr, n = noise_local.shape
    imfs = np.zeros((num_imfs, n), dtype=np.float64)
    o = OracleOpts()
    lib().oracle_default_opts(ctypes.byref(o))
    o.noise_sift_cap = noise_sift_cap
    o.solver, o.chunk, o.threads = solver, chunk, threads
    iters = np.zeros(2 * (num_imfs - 1), dtype=np.int32)
    o.iters_out = _i(iters)

    def arr(p, k):
        return np.ctypeslib.as_array(p, shape=(k,))

    sp = _Split()
    sp.nr_total, sp.rank, sp.world, sp.ctx = nr_total, rank, world, None
    sp.all_finished = _Split._fields_[4][1](lambda c, v: 1 if ops.all_finished(bool(v)) else 0)
    sp.recv_partial = _Split._fields_[5][1](lambda c, p, k: ops.recv_partial(arr(p, k)))
    sp.send_partial = _Split._fields_[6][1](lambda c, p, k: ops.send_partial(arr(p, k)))
    sp.broadcast_last = _Split._fields_[7][1](lambda c, p, k: ops.broadcast_last(arr(p, k)))
    f = lib().oracle_iceemdan_split_f64
    f.argtypes = [ctypes.c_size_t] * 4 + [_dp, _dp, ctypes.c_double, _dp,
                                          ctypes.POINTER(OracleOpts), ctypes.POINTER(_Split)]
    f.restype = ctypes.c_int
    rc = f(nr, n, num_imfs, max_iter, _d(y), _d(noise_local), nstd, _d(imfs), ctypes.byref(o),
           ctypes.byref(sp))
    if rc != 0:
        raise ValueError(f"oracle_iceemdan_split_f64 rejected its arguments (code {rc})")
    return (imfs, iters) if return_iters else imfs


def extrema(h, kind):
    """Compacted knots (x int32, y f64) of the maxima (kind 0) or minima (kind 1)."""
    h = np.ascontiguousarray(h, dtype=np.float64)
    kx = np.zeros(h.size, dtype=np.int32)
    ky = np.zeros(h.size, dtype=np.float64)
    k = lib().oracle_extrema_f64(_d(h), h.size, kind, _i(kx), _d(ky))
    return kx[:k].copy(), ky[:k].copy()


def boundary(kx, ky, kind):
    kx = np.ascontiguousarray(kx, dtype=np.int32)
    ky = np.array(ky, dtype=np.float64, copy=True)
    lib().oracle_boundary_f64(kx.size, _i(kx), _d(ky), kind)
    return ky


def spline_solve(kx, ky, solver=0, chunk=16):
    kx = np.ascontiguousarray(kx, dtype=np.int32)
    ky = np.ascontiguousarray(ky, dtype=np.float64)
    c = np.zeros(kx.size, dtype=np.float64)
    lib().oracle_spline_solve_f64(kx.size, _i(kx), _d(ky), _d(c), solver, chunk)
    return c


def spline_eval(n, kx, ky, c):
    kx = np.ascontiguousarray(kx, dtype=np.int32)
    ky = np.ascontiguousarray(ky, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    env = np.zeros(n, dtype=np.float64)
    lib().oracle_spline_eval_f64(n, kx.size, _i(kx), _d(ky), _d(c), _d(env))
    return env


def envelope(h, kind, solver=0, chunk=16):
    """Upper (kind 0) or lower (kind 1) envelope of h, as one sift iteration builds it."""
    kx, ky = extrema(h, kind)
    ky = boundary(kx, ky, kind)
    c = spline_solve(kx, ky, solver, chunk)
    return spline_eval(h.size, kx, ky, c)


def canonical_sum(v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().oracle_canonical_sum_f64(_d(v), v.size)


def canonical_sqdev(v, mean):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().oracle_canonical_sqdev_f64(_d(v), v.size, mean)


def tridiag_partitioned(l, m, u, r, chunk=16):
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (l, m, u, r)]
    x = np.zeros(arrs[0].size, dtype=np.float64)
    lib().oracle_tridiag_partitioned_f64(arrs[0].size, *[_d(a) for a in arrs], _d(x), chunk)
    return x


class Tape:
    """Oracle forward decomposition with its frozen structure recorded (knots, end-rule
    choices, marks, iteration counts, noise modes, stage statistics).

    ``imfs`` holds the forward result; ``replay(y)`` evaluates the decomposition at another
    input with that structure frozen (the map finite differences are taken of) and
    ``vjp(g)`` returns (d imfs / d y)^T g."""

    def __init__(self, y, noise, num_imfs, max_iter, nstd, *, solver=0, chunk=16, threads=0,
                 noise_sift_cap=2000, sd=0.05, sd2=0.5, tol=0.05, noise_from=None):
        """noise_from: another Tape of the same length, noise and options whose noise phase
        is reused (noise may then be None); the result equals a full call's."""
        self._h = None
        y = np.ascontiguousarray(y, dtype=np.float64)
        if noise_from is not None:
            self.nr, self.n = noise_from.nr, noise_from.n
        else:
            noise = np.ascontiguousarray(noise, dtype=np.float64)
            self.nr, self.n = noise.shape
        self.num_imfs = num_imfs
        self.imfs = np.zeros((num_imfs, self.n), dtype=np.float64)
        o = OracleOpts()
        lib().oracle_default_opts(ctypes.byref(o))
        o.noise_sift_cap = noise_sift_cap
        o.sd, o.sd2, o.tol = sd, sd2, tol
        o.solver, o.chunk, o.threads = solver, chunk, threads
        if noise_from is not None:
            h = lib().oracle_tape_forward_shared_f64(self.nr, self.n, num_imfs, max_iter, _d(y),
                                                     nstd, _d(self.imfs), ctypes.byref(o),
                                                     noise_from._h)
        else:
            h = lib().oracle_tape_forward_f64(self.nr, self.n, num_imfs, max_iter, _d(y),
                                              _d(noise), nstd, _d(self.imfs), ctypes.byref(o))
        if not h:
            raise ValueError("oracle_tape_forward_f64 rejected its arguments")
        self._h = h

    def replay(self, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros((self.num_imfs, self.n), dtype=np.float64)
        if lib().oracle_tape_replay_f64(self._h, _d(y), _d(out)) != 0:
            raise ValueError("replay failed")
        return out

    def vjp(self, gimfs):
        g = np.ascontiguousarray(gimfs, dtype=np.float64)
        assert g.shape == (self.num_imfs, self.n)
        gy = np.zeros(self.n, dtype=np.float64)
        lib().oracle_tape_vjp_f64(self._h, _d(g), _d(gy))
        return gy

    def vjp_recompute(self, gimfs):
        """vjp with every stage re-computed from its checkpoint (checkpoint-and-recompute)."""
        g = np.ascontiguousarray(gimfs, dtype=np.float64)
        assert g.shape == (self.num_imfs, self.n)
        gy = np.zeros(self.n, dtype=np.float64)
        lib().oracle_tape_vjp_recompute_f64(self._h, _d(g), _d(gy))
        return gy

    def recompute_mismatches(self):
        return lib().oracle_tape_recompute_mismatches(self._h)

    def iterations(self):
        return [lib().oracle_tape_iterations(self._h, i) for i in range(self.num_imfs - 1)]

    def step(self, stage, it, r, e):
        """(knot positions, end-rule flags, mark) of one recorded iteration."""
        kx = np.zeros(self.n, dtype=np.int32)
        bf, mk = ctypes.c_int(0), ctypes.c_int(0)
        k = lib().oracle_tape_step(self._h, stage, it, r, e, _i(kx), ctypes.byref(bf),
                                   ctypes.byref(mk))
        if k < 0:
            raise IndexError("no such step")
        return kx[:k].copy(), bf.value, mk.value

    def __del__(self):
        if self._h:
            lib().oracle_tape_free(self._h)
            self._h = None
