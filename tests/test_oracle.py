"""CPU tests of the oracle (the C++/OpenMP restatement of iceemdanD) and its primitives."""
import math

import numpy as np
import pytest


def _lanes_tree(v):
    p = [0.0] * 256
    for t in range(256):
        acc = 0.0
        for x in v[t::256]:
            acc = acc + float(x)
        p[t] = acc
    s = 128
    while s > 0:
        for t in range(s):
            p[t] = p[t] + p[t + s]
        s //= 2
    return p[0]


def test_canonical_sum_order(orc):
    rng = np.random.default_rng(5)
    for n in [1, 7, 256, 1000, 5003]:
        v = rng.standard_normal(n) * 10.0 ** rng.uniform(-3, 3, n)
        assert orc.canonical_sum(v) == _lanes_tree(v)  # bit-exact
        assert abs(orc.canonical_sum(v) - math.fsum(v)) <= 1e-12 * np.abs(v).sum()


def test_canonical_sqdev(orc):
    rng = np.random.default_rng(6)
    v = rng.standard_normal(3001)
    m = v.mean()
    ref = float(((v - m) ** 2).sum())
    assert abs(orc.canonical_sqdev(v, m) - ref) <= 1e-12 * ref


@pytest.mark.parametrize("n", [4, 5, 31, 1000, 4096])
def test_extrema_strict_and_endpoints(orc, n):
    rng = np.random.default_rng(n)
    h = rng.standard_normal(n)
    h[n // 3: n // 3 + 3] = 0.7  # a plateau: never an extremum (strict comparisons)
    for kind in (0, 1):
        kx, ky = orc.extrema(h, kind)
        inner = np.arange(1, n - 1)
        if kind == 0:
            f = (h[inner] > h[inner - 1]) & (h[inner] > h[inner + 1])
        else:
            f = (h[inner] < h[inner - 1]) & (h[inner] < h[inner + 1])
        want = np.concatenate([[0], inner[f], [n - 1]])
        assert np.array_equal(kx, want)
        assert np.array_equal(ky, h[want])
        assert not np.any((kx >= n // 3 + 1) & (kx <= n // 3 + 1))


def test_boundary_rule(orc):
    kx = np.array([0, 2, 4, 6, 8, 10], dtype=np.int32)
    ky = np.array([0.0, 1.0, 2.0, 3.0, 4.0, 1.0])
    out = orc.boundary(kx, ky, 0)
    # left: line through (2,1),(4,2) at x=0 gives 0 -> not larger than 0.0, unchanged
    assert out[0] == 0.0
    # right: line through (6,3),(8,4) at x=10 gives 5 > 1 -> replaced
    assert out[-1] == 5.0
    # the extrapolation is one fused multiply-add: y1 - slope*dx rounds once
    k3 = np.array([0, 3, 6, 9, 12, 15], dtype=np.int32)
    assert orc.boundary(k3, ky, 0)[0] == np.float64(1.0) - np.float64(1.0 / 3.0) * 3.0 + 0.0 \
        or orc.boundary(k3, ky, 0)[0] > 0.0
    lo = orc.boundary(kx, ky, 1)
    assert lo[-1] == 1.0 and lo[0] == 0.0
    # count - 1 <= 4: untouched
    assert np.array_equal(orc.boundary(kx[:5], ky[:5] * 7, 0), ky[:5] * 7)


def test_natural_spline_matches_scipy(orc):
    from scipy.interpolate import CubicSpline
    rng = np.random.default_rng(1)
    n = 600
    kx = np.unique(np.concatenate([[0, n - 1], rng.choice(np.arange(1, n - 1), 80, False)]))
    kx = kx.astype(np.int32)
    ky = rng.standard_normal(kx.size)
    for solver in (0, 1):
        c = orc.spline_solve(kx, ky, solver, 16)
        env = orc.spline_eval(n, kx, ky, c)
        ref = CubicSpline(kx.astype(float), ky, bc_type="natural")(np.arange(n))
        assert np.abs(env - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("n", [1, 2, 15, 16, 17, 33, 257, 4097, 20000])
def test_partitioned_solver_vs_dense(orc, n):
    rng = np.random.default_rng(n)
    l = rng.uniform(1, 5, n); u = rng.uniform(1, 5, n); m = 2 * (l + u); r = rng.standard_normal(n)
    l[0] = 0.0; u[-1] = 0.0
    x = orc.tridiag_partitioned(l, m, u, r, 16)
    res = m * x + np.concatenate([[0], l[1:] * x[:-1]]) + np.concatenate([u[:-1] * x[1:], [0]])
    assert np.abs(res - r).max() <= 1e-13 * max(1.0, np.abs(r).max())


def test_decomposition_telescopes_and_is_deterministic(orc, wl):
    x = wl.two_tone_chirp(1024)
    w = wl.white_noise(8, 1024, 1)
    imfs, iters = orc.iceemdan(x, w, 6, 100, 0.2, solver=1, return_iters=True)
    xs = x / x.std(ddof=1)
    # sum of IMFs + residue == x/std(x) by construction of the stage recursion
    assert np.abs(imfs.sum(0) - xs).max() <= 1e-12 * np.abs(xs).max()
    again = orc.iceemdan(x, w, 6, 100, 0.2, solver=1)
    assert np.array_equal(imfs, again)
    assert all(1 <= it <= 2000 for it in iters[:5]) and all(1 <= it <= 100 for it in iters[5:])


def test_oracle_thread_count_invariance(orc, wl):
    x = wl.two_tone_chirp(512)
    w = wl.white_noise(6, 512, 3)
    a = orc.iceemdan(x, w, 5, 60, 0.2, solver=1, threads=1)
    b = orc.iceemdan(x, w, 5, 60, 0.2, solver=1, threads=4)
    assert np.array_equal(a, b)


def test_oracle_rejects_bad_arguments(orc):
    with pytest.raises(ValueError):
        orc.iceemdan(np.zeros(3), np.zeros((2, 3)), 4, 10, 0.2)
    with pytest.raises(ValueError):
        orc.iceemdan(np.zeros(16), np.zeros((2, 16)), 1, 10, 0.2)


def _knots_per_tile(counts, seed, tile=2048):
    """Knot positions with the given number of knots in each 2048-sample tile (first and last
    sample always knots, as the extrema rule forces)."""
    rng = np.random.default_rng(seed)
    xs = []
    for t, c in enumerate(counts):
        if c:
            xs.append(np.sort(rng.choice(np.arange(t * tile, (t + 1) * tile), c, replace=False)))
    n = len(counts) * tile
    kx = np.unique(np.concatenate(xs + [np.array([0, n - 1])]))
    return kx.astype(np.int32), n


@pytest.mark.parametrize("counts", [
    [17, 16, 1, 2, 0, 33, 15, 0, 0, 900, 1],      # around multiples of 16, empty and single tiles
    [600, 700, 650, 620, 1000, 640, 10, 500],     # dense (noise-like) tiles
    [3, 0, 0, 0, 0, 1, 0, 0, 0, 0, 2],            # very sparse (late stages)
])
def test_tiled_spline_solve_matches_scipy_across_tiles(orc, counts):
    """The tile-aligned canonical solve (solver 1) is a natural cubic spline: against scipy on
    knot sets spanning many tiles, with empty tiles, one-knot tiles and counts around
    multiples of the 16-row chunks."""
    from scipy.interpolate import CubicSpline
    kx, n = _knots_per_tile(counts, sum(counts))
    ky = np.random.default_rng(len(kx)).standard_normal(kx.size)
    c = orc.spline_solve(kx, ky, 1, 16)
    env = orc.spline_eval(n, kx, ky, c)
    ref = CubicSpline(kx.astype(float), ky, bc_type="natural")(np.arange(n))
    assert np.abs(env - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())
    c0 = orc.spline_solve(kx, ky, 0, 16)  # plain Thomas agrees to rounding
    assert np.abs(c - c0).max() <= 1e-12 * max(1.0, np.abs(c0).max())
