"""GPU parity: the CUDA engine against the CPU oracle on identical inputs.

Every floating-point step of the engine follows one canonical order that the oracle evaluates
too (solver=1, chunk=16), so the expected result is bit-identical.  The decomposition is
checked against the oracle's solver 1; where a tolerance is written, it is the 1e-9 max
relative IMF error the FP64 path is held to.
"""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHUNK = 16
IMF_RTOL = 1e-9


def _torch():
    import torch
    return torch


def _h(nr, n, seed, plateau=True):
    rng = np.random.default_rng(seed)
    h = rng.standard_normal((nr, n))
    if plateau and n > 20:
        h[:, n // 2: n // 2 + 4] = 0.25
        h[0, 1:4] = [0.5, 0.5, 0.5]
    return h


SIZES = [5, 100, 2047, 2048, 2049, 5000, 30001]


@pytest.mark.parametrize("n", SIZES)
def test_extrema_bitexact(pkg, orc, cuda, n):
    torch = _torch()
    h = _h(3, n, n)
    kxM, kyM, kxm, kym, cnt = pkg.extrema(torch.tensor(h, device=cuda))
    kxM, kyM, kxm, kym, cnt = (t.cpu().numpy() for t in (kxM, kyM, kxm, kym, cnt))
    for r in range(3):
        for kind, (kx, ky) in enumerate(((kxM, kyM), (kxm, kym))):
            ox, oy = orc.extrema(h[r], kind)
            oy = orc.boundary(ox, oy, kind)
            k = cnt[kind, r]
            assert k == ox.size
            assert np.array_equal(kx[r, :k], ox)
            assert np.array_equal(ky[r, :k], oy)


@pytest.mark.parametrize("n", SIZES + [244032])
def test_envelopes_bitexact(pkg, orc, cuda, n):
    torch = _torch()
    nr = 2 if n < 100000 else 1
    h = _h(nr, n, 7 * n)
    up, lo, cnt = pkg.envelopes(torch.tensor(h, device=cuda))
    up, lo = up.cpu().numpy(), lo.cpu().numpy()
    for r in range(nr):
        assert np.array_equal(up[r], orc.envelope(h[r], 0, solver=1, chunk=CHUNK))
        assert np.array_equal(lo[r], orc.envelope(h[r], 1, solver=1, chunk=CHUNK))


def test_envelopes_smooth_signal(pkg, orc, cuda, wl):
    torch = _torch()
    x = wl.two_tone_chirp(4096)[None, :]
    up, lo, _ = pkg.envelopes(torch.tensor(x, device=cuda))
    assert np.array_equal(up.cpu().numpy()[0], orc.envelope(x[0], 0, solver=1))
    assert np.array_equal(lo.cpu().numpy()[0], orc.envelope(x[0], 1, solver=1))


@pytest.mark.parametrize("n", [1, 2, 16, 17, 300, 5000, 70000])
def test_tridiag_bitexact(pkg, orc, cuda, n):
    torch = _torch()
    rng = np.random.default_rng(n)
    l = rng.uniform(1, 9, (2, n)); u = rng.uniform(1, 9, (2, n)); m = 2 * (l + u) + 0.5
    r = rng.standard_normal((2, n))
    l[:, 0] = 0.0; u[:, -1] = 0.0
    x = pkg.tridiag(*(torch.tensor(a, device=cuda) for a in (l, m, u, r))).cpu().numpy()
    for b in range(2):
        assert np.array_equal(x[b], orc.tridiag_partitioned(l[b], m[b], u[b], r[b], CHUNK))


def test_canonical_sums_bitexact(pkg, orc, cuda):
    torch = _torch()
    rng = np.random.default_rng(3)
    for n in [1, 255, 256, 4097, 244032]:
        v = rng.standard_normal((3, n)) * 3.0 + 1.0
        mean = v.mean(axis=1)
        s, q = pkg.canonical_sums(torch.tensor(v, device=cuda), torch.tensor(mean, device=cuda))
        s, q = s.cpu().numpy(), q.cpu().numpy()
        for b in range(3):
            assert s[b] == orc.canonical_sum(v[b])
            assert q[b] == orc.canonical_sqdev(v[b], mean[b])


def _rel_err(a, b):
    return float(np.max(np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)))


def _decompose_both(pkg, orc, cuda, x, noise, nimf, max_iter, nstd=0.2, cap=2000):
    torch = _torch()
    imfs, iters = pkg.iceemdan(torch.tensor(x, device=cuda), noise.shape[0], nimf, max_iter, nstd,
                               noise=torch.tensor(noise, device=cuda), noise_sift_cap=cap,
                               return_iters=True)
    ref, riters = orc.iceemdan(x, noise, nimf, max_iter, nstd, solver=1, chunk=CHUNK,
                               noise_sift_cap=cap, return_iters=True)
    return imfs.cpu().numpy(), list(iters), ref, list(riters)


def test_decomposition_small_bitexact(pkg, orc, cuda, wl):
    x = wl.two_tone_chirp(1024)
    noise = wl.white_noise(8, 1024, 1)
    got, it, ref, rit = _decompose_both(pkg, orc, cuda, x, noise, 6, 100)
    assert it == rit
    assert np.array_equal(got, ref)


def test_decomposition_ragged_tiles(pkg, orc, cuda, wl):
    # n not a multiple of the 2048-sample tile, several tiles, eeg-like content
    x = wl.eeg_like(5000, seed=11)
    noise = wl.white_noise(6, 5000, 12)
    got, it, ref, rit = _decompose_both(pkg, orc, cuda, x, noise, 5, 80, cap=300)
    assert it == rit
    assert _rel_err(got, ref) <= IMF_RTOL
    assert np.array_equal(got, ref)


def test_decomposition_config1(pkg, orc, cuda, wl):
    """Plain ICEEMDAN at N=4096, NR=50, MaxIter=300, 12 IMFs (two tones + chirp + noise)."""
    x = wl.two_tone_chirp(4096, seed=0)
    noise = wl.white_noise(50, 4096, 1)
    got, it, ref, rit = _decompose_both(pkg, orc, cuda, x, noise, 12, 300)
    assert it == rit
    assert _rel_err(got, ref) <= IMF_RTOL
    assert np.array_equal(got, ref)
    xs = x / x.std(ddof=1)
    assert np.abs(got.sum(0) - xs).max() <= 1e-12 * np.abs(xs).max()


def _curand_device_normals(count, seed, device):
    """N(0,1) doubles from cuRAND's device generator (CURAND_RNG_PSEUDO_DEFAULT = XORWOW),
    the call cudaICEEMDAN.cu:1460-1462 makes."""
    torch = _torch()
    lib = ctypes.CDLL("libcurand.so.10") if os.path.exists("/usr/local/cuda/lib64/libcurand.so.10") \
        else ctypes.CDLL("libcurand.so")
    gen = ctypes.c_void_p()
    assert lib.curandCreateGenerator(ctypes.byref(gen), 100) == 0  # PSEUDO_DEFAULT
    assert lib.curandSetPseudoRandomGeneratorSeed(gen, ctypes.c_ulonglong(seed)) == 0
    out = torch.empty(count + (count & 1), dtype=torch.float64, device=device)
    assert lib.curandGenerateNormalDouble(gen, ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_size_t(out.numel()), ctypes.c_double(0.0),
                                          ctypes.c_double(1.0)) == 0
    torch.cuda.synchronize()
    lib.curandDestroyGenerator(gen)
    return out[:count]


def test_dropin_iceemdanD_raw_pointers(pkg, orc, cuda, wl):
    """The reference-shaped entry point: raw device pointers, internal cuRAND seed 1234."""
    torch = _torch()
    n, nr, nimf, mi = 2000, 10, 6, 120
    x = wl.two_tone_chirp(n, seed=4)
    d_y = torch.tensor(x, device=cuda)
    d_x = torch.arange(n, dtype=torch.int32, device=cuda)
    d_imfs = torch.full((nimf, n), float("nan"), dtype=torch.float64, device=cuda)
    secs = pkg.iceemdanD(nr, n, nimf, mi, d_x.data_ptr(), d_y.data_ptr(), d_imfs.data_ptr(), 0.2)
    assert secs > 0.0
    noise = _curand_device_normals(nr * n, 1234, cuda).reshape(nr, n).cpu().numpy()
    ref = orc.iceemdan(x, noise, nimf, mi, 0.2, solver=1, chunk=CHUNK)
    assert np.array_equal(d_imfs.cpu().numpy(), ref)


def test_curand_host_generator_matches_device(cuda):
    """The cuRAND host generator (usable without a GPU) reproduces the device stream to within
    2 ulps, not bit for bit (its Box-Muller uses the host math library): parity tests use
    device-generated noise."""
    lib = ctypes.CDLL("libcurand.so.10")
    dev = _curand_device_normals(65536, 1234, cuda).cpu().numpy()
    gen = ctypes.c_void_p()
    assert lib.curandCreateGeneratorHost(ctypes.byref(gen), 100) == 0
    assert lib.curandSetPseudoRandomGeneratorSeed(gen, ctypes.c_ulonglong(1234)) == 0
    host = np.zeros(65536)
    assert lib.curandGenerateNormalDouble(gen, host.ctypes.data_as(ctypes.c_void_p),
                                          ctypes.c_size_t(65536), ctypes.c_double(0.0),
                                          ctypes.c_double(1.0)) == 0
    lib.curandDestroyGenerator(gen)
    mism = int(np.count_nonzero(host != dev))
    print("host/device normals differing:", mism, "max abs diff:", float(np.max(np.abs(host - dev))))
    assert np.max(np.abs(host - dev)) <= 1e-15 * np.max(np.abs(dev))


def test_coordinates_must_be_sample_index(pkg, cuda):
    torch = _torch()
    n = 256
    d_y = torch.randn(n, dtype=torch.float64, device=cuda)
    d_x = torch.arange(n, dtype=torch.int32, device=cuda) * 2
    d_imfs = torch.empty((3, n), dtype=torch.float64, device=cuda)
    with pytest.raises(pkg.CeemdanError) as ei:
        pkg.iceemdanD(4, n, 3, 10, d_x.data_ptr(), d_y.data_ptr(), d_imfs.data_ptr(), 0.2)
    assert ei.value.status == 2


def _curand_device_normals_f32(count, seed, device):
    """N(0,1) floats from cuRAND's device generator (curandGenerateNormal, the FP32 reference
    path's call, cudaICEEMDAN.cu:741), widened to float64."""
    torch = _torch()
    lib = ctypes.CDLL("libcurand.so.10") if os.path.exists("/usr/local/cuda/lib64/libcurand.so.10") \
        else ctypes.CDLL("libcurand.so")
    gen = ctypes.c_void_p()
    assert lib.curandCreateGenerator(ctypes.byref(gen), 100) == 0  # PSEUDO_DEFAULT
    assert lib.curandSetPseudoRandomGeneratorSeed(gen, ctypes.c_ulonglong(seed)) == 0
    out = torch.empty(count + (count & 1), dtype=torch.float32, device=device)
    assert lib.curandGenerateNormal(gen, ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_size_t(out.numel()), ctypes.c_float(0.0),
                                    ctypes.c_float(1.0)) == 0
    torch.cuda.synchronize()
    lib.curandDestroyGenerator(gen)
    return out[:count].double()


def test_dropin_iceemdanS_float(pkg, orc, cuda, wl):
    """The FP32 drop-in (cudaICEEMDAN.cuh:25): float data and IMFs, cuRAND float normals seed
    1234; computed in FP64 on the widened data, so the result is the oracle's FP64 result
    rounded to float."""
    torch = _torch()
    n, nr, nimf, mi = 2000, 10, 6, 120
    x = wl.two_tone_chirp(n, seed=4).astype(np.float32)
    d_y = torch.tensor(x, device=cuda)
    d_x = torch.arange(n, dtype=torch.int32, device=cuda)
    d_imfs = torch.full((nimf, n), float("nan"), dtype=torch.float32, device=cuda)
    secs = pkg.iceemdanS(nr, n, nimf, mi, d_x.data_ptr(), d_y.data_ptr(), d_imfs.data_ptr(), 0.2)
    assert secs > 0.0
    noise = _curand_device_normals_f32(nr * n, 1234, cuda).reshape(nr, n).cpu().numpy()
    ref = orc.iceemdan(x.astype(np.float64), noise, nimf, mi, float(np.float32(0.2)), solver=1,
                       chunk=CHUNK)
    assert np.array_equal(d_imfs.cpu().numpy(), ref.astype(np.float32))


def test_tensor_api_float32_with_external_noise(pkg, orc, cuda, wl):
    torch = _torch()
    n, nr = 1500, 6
    x = wl.eeg_like(n, seed=5).astype(np.float32)
    noise = wl.white_noise(nr, n, 6)
    got = pkg.iceemdan(torch.tensor(x, device=cuda), nr, 5, 80, 0.2,
                       noise=torch.tensor(noise, device=cuda), noise_sift_cap=200)
    assert got.dtype == torch.float32
    ref = orc.iceemdan(x.astype(np.float64), noise, 5, 80, float(np.float32(0.2)), solver=1,
                       chunk=CHUNK, noise_sift_cap=200)
    assert np.array_equal(got.cpu().numpy(), ref.astype(np.float32))


def _edge_signal(kind, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "noise":
        return rng.standard_normal(n)
    if kind == "plateaus":  # runs of equal samples: non-strict extrema, zero slopes
        return np.repeat(rng.standard_normal((n + 3) // 4), 4)[:n]
    if kind == "steps":  # integer-valued walk: many exact ties between neighbours
        return np.cumsum(rng.integers(-1, 2, n)).astype(np.float64)
    if kind == "tiny":  # values near the bottom of the normal range
        return rng.standard_normal(n) * 1e-300
    raise ValueError(kind)


EDGE_CASES = [
    # (kind, n, nr, nimf, max_iter, cap)
    ("noise", 4, 1, 2, 1, 5),
    ("noise", 5, 3, 3, 7, 20),
    ("noise", 17, 2, 3, 50, 100),
    ("plateaus", 2047, 3, 4, 30, 60),
    ("noise", 2049, 1, 5, 40, 80),
    ("steps", 4097, 4, 5, 40, 80),
    ("plateaus", 6145, 2, 6, 25, 50),
    ("tiny", 3000, 3, 4, 30, 60),
    ("noise", 1, 1, 2, 1, 1),  # rejected: n < 4
]


@pytest.mark.parametrize("kind,n,nr,nimf,mi,cap", EDGE_CASES)
def test_edge_shapes_bitexact(pkg, orc, cuda, kind, n, nr, nimf, mi, cap):
    """Shapes and values at the edges: minimum and odd lengths, lengths around the 2048-sample
    tiles, one realization, one sift iteration, plateaus, integer ties, values near underflow.
    The engine equals the oracle bit for bit (NaN where the oracle has NaN)."""
    torch = _torch()
    x = _edge_signal(kind, n, n + nr)
    noise = np.random.default_rng(7 * n + nr).standard_normal((nr, n))
    if n < 4:
        with pytest.raises(pkg.CeemdanError):
            pkg.iceemdan(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2,
                         noise=torch.tensor(noise, device=cuda), noise_sift_cap=cap)
        return
    got, it, ref, rit = _decompose_both(pkg, orc, cuda, x, noise, nimf, mi, cap=cap)
    assert it == rit
    assert np.array_equal(got, ref, equal_nan=True)


def test_constant_signal_matches_oracle(pkg, orc, cuda):
    """std(x) = 0: the standardisation divides by zero as in the reference; whatever values
    follow, engine and oracle agree (NaN-aware)."""
    torch = _torch()
    n, nr = 1000, 2
    x = np.full(n, 3.0)
    noise = np.random.default_rng(1).standard_normal((nr, n))
    got, it, ref, rit = _decompose_both(pkg, orc, cuda, x, noise, 3, 10, cap=20)
    assert it == rit
    assert np.array_equal(got, ref, equal_nan=True)


def test_batch_entry_equals_single_calls(pkg, cuda, wl):
    """ceemdan_batch_f64: ragged channels on 3 internal streams equal one plain call each (seed
    + channel index), bit for bit."""
    torch = _torch()
    lengths = [5000, 1200, 8191, 2048]
    ys = [torch.tensor(wl.eeg_like(n, seed=40 + i), device=cuda) for i, n in enumerate(lengths)]
    got = pkg.iceemdan_batch(ys, 12, 5, 40, 0.2, seed=77, streams=3, noise_sift_cap=100)
    for i, y in enumerate(ys):
        ref = pkg.iceemdan(y, 12, 5, 40, 0.2, seed=77 + i, noise_sift_cap=100)
        assert torch.equal(got[i], ref)


def test_shared_noise_state_equals_full_calls(pkg, orc, cuda, wl):
    """The noise phase depends only on the noise: a second channel of the same length started
    from the first channel's noise-phase state equals its full decomposition bit for bit, and
    so does the oracle's."""
    torch = _torch()
    n, nr, nimf, mi = 3000, 8, 6, 60
    xa = wl.eeg_like(n, seed=31)
    xb = wl.two_tone_chirp(n, seed=32)
    kw = dict(noise_sift_cap=120, seed=99, return_iters=True)
    _, _, modes, state = pkg.iceemdan(torch.tensor(xa, device=cuda), nr, nimf, mi, 0.2,
                                      return_noise_modes=True, return_noise_state=True, **kw)
    assert torch.equal(state[:nimf * nr * n].view(nimf, nr, n), modes)
    full, it_full = pkg.iceemdan(torch.tensor(xb, device=cuda), nr, nimf, mi, 0.2, **kw)
    fast, it_fast = pkg.iceemdan(torch.tensor(xb, device=cuda), nr, nimf, mi, 0.2,
                                 noise_state=state, **kw)
    assert torch.equal(full, fast)
    assert it_fast[:nimf - 1] == [0] * (nimf - 1) and it_fast[nimf - 1:] == it_full[nimf - 1:]
    import ceemdan_gpu_b200.multichannel as mc
    shared = mc.decompose_shared_noise(pkg, [xa, xb], nr, nimf, mi, 0.2, seed=99, device=cuda,
                                       noise_sift_cap=120)
    assert torch.equal(shared[1], full)


def test_noise_cache_reuses_the_noise_phase(pkg, cuda, wl):
    """With the noise-phase cache on, a second channel of the same length and seed skips the
    noise phase (its noise iteration counts are 0) and equals the uncached result bit for bit;
    another length misses and recomputes."""
    torch = _torch()
    L = pkg.lib()
    n, nr, nimf, mi = 2500, 6, 5, 50
    kw = dict(noise_sift_cap=100, seed=5, return_iters=True)
    xa = torch.tensor(wl.eeg_like(n, seed=61), device=cuda)
    xb = torch.tensor(wl.two_tone_chirp(n, seed=62), device=cuda)
    prev = L.ceemdan_noise_cache(0)
    try:
        ref_b, it_ref = pkg.iceemdan(xb, nr, nimf, mi, 0.2, **kw)  # uncached
        L.ceemdan_noise_cache(1 << 30)
        _, it_a = pkg.iceemdan(xa, nr, nimf, mi, 0.2, **kw)  # fills the cache
        assert it_a[:nimf - 1] != [0] * (nimf - 1)
        got_b, it_b = pkg.iceemdan(xb, nr, nimf, mi, 0.2, **kw)  # hits
        assert it_b[:nimf - 1] == [0] * (nimf - 1)
        assert torch.equal(got_b, ref_b) and it_b[nimf - 1:] == it_ref[nimf - 1:]
        xc = torch.tensor(wl.eeg_like(n + 1, seed=63), device=cuda)
        _, it_c = pkg.iceemdan(xc, nr, nimf, mi, 0.2, **kw)  # other length: misses
        assert it_c[:nimf - 1] != [0] * (nimf - 1)
    finally:
        L.ceemdan_noise_cache(0)
        L.ceemdan_noise_cache(prev)
