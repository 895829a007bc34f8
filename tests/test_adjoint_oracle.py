"""The oracle's reverse pass (frozen structure) against central finite differences.

With the knot positions, end-rule choices, stale-mean choices, marks and iteration counts of
a recorded forward call frozen, the decomposition is a differentiable map y -> imfs; the
oracle's replay evaluates that map and its vjp is (d imfs / d y)^T g.  These CPU tests pin the
vjp (the checker of the CUDA backward entry) with central differences, eps = 1e-6, on the
weighted-energy loss sum_k w_k |IMF_k|^2, w_k ~ U(0, 1) from seed 4."""
import numpy as np
import pytest


def _loss_fd(tape, x, w, coords, eps=1e-6):
    def L(y):
        return float(np.sum(w[:, None] * tape.replay(y) ** 2))
    out = []
    for k in coords:
        e = np.zeros_like(x)
        e[k] = eps
        out.append((L(x + e) - L(x - e)) / (2 * eps))
    return np.array(out)


def _case(wl, n, nr, seed=0):
    x = wl.two_tone_chirp(n, seed=seed)
    noise = np.random.default_rng(seed + 1).standard_normal((nr, n))
    return x, noise


@pytest.mark.parametrize("solver", [0, 1])
def test_tape_forward_and_replay_are_the_forward(orc, wl, solver):
    x, noise = _case(wl, 1500, 4)
    ref = orc.iceemdan(x, noise, 6, 30, 0.2, solver=solver, noise_sift_cap=60)
    t = orc.Tape(x, noise, 6, 30, 0.2, solver=solver, noise_sift_cap=60)
    assert np.array_equal(t.imfs, ref)
    assert np.array_equal(t.replay(x), ref)
    its = t.iterations()
    assert len(its) == 5 and min(its) >= 1
    # recorded knots include both end samples and increase strictly
    kx, bf, mk = t.step(0, 0, 0, 0)
    assert kx[0] == 0 and kx[-1] == x.size - 1 and np.all(np.diff(kx) > 0)


@pytest.mark.parametrize("solver", [0, 1])
def test_vjp_matches_central_differences(orc, wl, solver):
    """256 random coordinates, as the differentiation workload checks them (there with
    N=8192, NR=50, MaxIter=100 per signal; here a smaller signal so that the 512 replays
    take seconds)."""
    x, noise = _case(wl, 2048, 6)
    nimf = 8
    t = orc.Tape(x, noise, nimf, 100, 0.2, solver=solver, noise_sift_cap=200)
    w = np.random.default_rng(4).uniform(size=nimf)
    gy = t.vjp(2.0 * w[:, None] * t.imfs)
    coords = np.random.default_rng(5).choice(x.size, 256, replace=False)
    fd = _loss_fd(t, x, w, coords)
    scale = np.abs(gy).max()
    assert np.abs(fd - gy[coords]).max() <= 1e-6 * scale
    # random directions (every coordinate at once)
    rng = np.random.default_rng(6)
    for _ in range(2):
        v = rng.standard_normal(x.size)
        eps = 1e-6
        Lp = np.sum(w[:, None] * t.replay(x + eps * v) ** 2)
        Lm = np.sum(w[:, None] * t.replay(x - eps * v) ** 2)
        fdv = (Lp - Lm) / (2 * eps)
        assert abs(fdv - gy @ v) <= 1e-6 * abs(gy) @ abs(v)


def _per_coordinate(tape, x, w, gy, coords, eps):
    fd = _loss_fd(tape, x, w, coords, eps)
    return np.abs(fd - gy[coords]) / np.abs(gy[coords])


def test_vjp_per_coordinate_relative_error(orc, wl):
    """Per-coordinate relative error |fd - g| / |g| on 128 random coordinates.  With
    eps = 1e-5 every coordinate agrees to 1e-6; at the differentiation workload's eps = 1e-6 the
    central difference itself carries the loss's rounding noise divided by eps (about 1e-9
    absolute here), so the bound there is 1e-6 for the median and 1e-5 for every coordinate."""
    x, noise = _case(wl, 2048, 6)
    nimf = 8
    t = orc.Tape(x, noise, nimf, 100, 0.2, solver=1, noise_sift_cap=200)
    w = np.random.default_rng(4).uniform(size=nimf)
    gy = t.vjp(2.0 * w[:, None] * t.imfs)
    coords = np.random.default_rng(7).choice(x.size, 128, replace=False)
    rel5 = _per_coordinate(t, x, w, gy, coords, 1e-5)
    rel6 = _per_coordinate(t, x, w, gy, coords, 1e-6)
    print("per-coordinate relative error, eps 1e-5: max", rel5.max(), "median",
          np.median(rel5), "; eps 1e-6: max", rel6.max(), "median", np.median(rel6))
    assert rel5.max() <= 1e-6
    assert np.median(rel6) <= 1e-6 and rel6.max() <= 1e-5


def test_vjp_at_differentiation_workload_size(orc, wl):
    """One signal of the differentiation workload (two-tone chirp seed 10, N = 8192, NR = 50,
    13 IMFs, MaxIter 100, noise sift cap 2000): per-coordinate relative error of the oracle's
    vjp against central differences (eps = 1e-5) on 16 random coordinates, each <= 1e-6."""
    x = wl.two_tone_chirp(8192, seed=10)
    noise = np.random.default_rng(1).standard_normal((50, 8192))
    nimf = 13
    t = orc.Tape(x, noise, nimf, 100, 0.2, solver=1, noise_sift_cap=2000)
    w = np.random.default_rng(4).uniform(size=nimf)
    gy = t.vjp(2.0 * w[:, None] * t.imfs)
    coords = np.random.default_rng(8).choice(x.size, 16, replace=False)
    rel = _per_coordinate(t, x, w, gy, coords, 1e-5)
    print("N=8192 NR=50: per-coordinate relative error max", rel.max(), "median",
          np.median(rel))
    assert rel.max() <= 1e-6


def test_vjp_through_stale_means_caps_and_end_rules(orc, wl):
    """Short signal (stages with <= 3 knots keep a stale mean envelope; < 6 knots skip the
    end rule) and a sift cap of 3 (every realization exports its mode at the cap)."""
    x, noise = _case(wl, 40, 3, seed=7)
    nimf = 5
    t = orc.Tape(x, noise, nimf, 3, 0.2, noise_sift_cap=50)
    stale = ends = capped = 0
    for s, J in enumerate(t.iterations()):
        assert J <= 3
        for j in range(J):
            for r in range(3):
                k0, b0, mk = t.step(s, j, r, 0)
                k1, b1, _ = t.step(s, j, r, 1)
                stale += (k0.size <= 3 or k1.size <= 3)
                ends += (b0 != 0 or b1 != 0)
                capped += (mk == 0 and j == 2)
    assert stale > 0 and ends > 0 and capped > 0
    w = np.random.default_rng(4).uniform(size=nimf)
    gy = t.vjp(2.0 * w[:, None] * t.imfs)
    coords = np.arange(x.size)
    fd = _loss_fd(t, x, w, coords)
    assert np.abs(fd - gy).max() <= 1e-6 * np.abs(gy).max()


def test_vjp_is_linear_in_the_cotangent(orc, wl):
    x, noise = _case(wl, 700, 3, seed=9)
    t = orc.Tape(x, noise, 5, 20, 0.2, noise_sift_cap=40)
    rng = np.random.default_rng(10)
    g1, g2 = rng.standard_normal((2, 5, x.size))
    a = t.vjp(1.5 * g1 - 0.25 * g2)
    b = 1.5 * t.vjp(g1) - 0.25 * t.vjp(g2)
    assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()
    assert np.array_equal(t.vjp(np.zeros((5, x.size))), np.zeros(x.size))


@pytest.mark.parametrize("n,nr,nimf,mi,cap", [(1024, 4, 6, 30, 60), (40, 3, 5, 3, 50)])
def test_stage_checkpoints_reproduce_the_structure(orc, wl, n, nr, nimf, mi, cap):
    """Checkpoint and recompute: a stage re-run from its input and the carries it started from
    (mean envelope, sifting fraction) reproduces every recorded step, and the vjp computed that
    way equals the full-tape vjp bit for bit."""
    x, noise = _case(wl, n, nr, seed=3)
    t = orc.Tape(x, noise, nimf, mi, 0.2, solver=1, noise_sift_cap=cap)
    assert t.recompute_mismatches() == 0
    g = np.random.default_rng(12).standard_normal((nimf, n))
    assert np.array_equal(t.vjp_recompute(g), t.vjp(g))


def test_vjp_across_tiles_on_an_eeg_like_signal(orc, wl):
    """EEG-shaped signal over three 2048-sample tiles (ragged last tile), tile-aligned
    canonical solve in the forward: central differences at 64 coordinates, with tile-boundary
    samples among them."""
    n, nr, nimf = 5000, 3, 7
    x = wl.eeg_like(n, seed=13)
    noise = np.random.default_rng(14).standard_normal((nr, n))
    t = orc.Tape(x, noise, nimf, 40, 0.2, solver=1, noise_sift_cap=80)
    w = np.random.default_rng(4).uniform(size=nimf)
    gy = t.vjp(2.0 * w[:, None] * t.imfs)
    coords = np.concatenate([[0, 2047, 2048, 4095, 4096, n - 1],
                             np.random.default_rng(15).choice(n, 58, replace=False)])
    fd = _loss_fd(t, x, w, coords)
    assert np.abs(fd - gy[coords]).max() <= 1e-6 * np.abs(gy).max()


def test_shared_noise_phase_gives_the_full_call(orc, wl):
    """A taped forward started from another signal's noise phase (same length, noise and
    options) equals a full call: IMFs, iteration counts and gradients bit for bit."""
    n, nr, nimf = 1500, 4, 6
    noise = np.random.default_rng(21).standard_normal((nr, n))
    first = orc.Tape(wl.two_tone_chirp(n, seed=1), noise, nimf, 40, 0.2, solver=1,
                     noise_sift_cap=80)
    x = wl.eeg_like(n, seed=22)
    full = orc.Tape(x, noise, nimf, 40, 0.2, solver=1, noise_sift_cap=80)
    shared = orc.Tape(x, None, nimf, 40, 0.2, solver=1, noise_sift_cap=80, noise_from=first)
    assert np.array_equal(shared.imfs, full.imfs)
    assert shared.iterations() == full.iterations()
    g = np.random.default_rng(23).standard_normal((nimf, n))
    assert np.array_equal(shared.vjp(g), full.vjp(g))
