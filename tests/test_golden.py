"""CPU: the oracle against golden outputs of the reference's own CUDA implementation
(tests/golden/*.npz, made by tests/golden/make_ref_fixtures.py from oracle/_ref)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_ref_fixtures import DEC_CASE, ENV_CASES, envelope_input  # noqa: E402


def _load(name):
    path = os.path.join(HERE, "golden", name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return np.load(path)


def test_oracle_envelopes_match_reference(orc):
    """One envelope pass: the reference's kernels + CUB + cuSPARSE vs the oracle: identical
    knot counts (strict-extrema sets), envelopes within 1e-12 (solver rounding)."""
    g = _load("ref_envelopes.npz")
    for nr, n, seed in ENV_CASES:
        h = envelope_input(nr, n, seed)
        for r in range(nr):
            for kind, env in ((0, g[f"up_{n}"][r]), (1, g[f"lo_{n}"][r])):
                kx, _ = orc.extrema(h[r], kind)
                assert kx.size == g[f"cnt_{n}"][kind, r]
                for solver in (0, 1):
                    want = orc.envelope(h[r], kind, solver=solver)
                    assert np.abs(env - want).max() <= 1e-12 * np.abs(want).max()


def _stats(imfs):
    e = (imfs ** 2).sum(axis=1)
    zc = (np.diff(np.signbit(imfs).astype(np.int8), axis=1) != 0).mean(axis=1)
    return e / e.sum(), zc


def test_oracle_decomposition_matches_reference_statistics(orc, wl):
    """Full decomposition on the reference's own noise: the reference telescopes exactly, and
    its per-IMF energy fractions and zero-crossing rates differ from the oracle's by no more
    than 3x the oracle's own spread between two exact tridiagonal solvers (the sifting is
    rounding-sensitive, so IMF samples themselves are not compared at 1e-9)."""
    g = _load("ref_iceemdan.npz")
    nr, n, nimf, mi, nstd = DEC_CASE
    x = wl.two_tone_chirp(n, seed=0)
    got = g["imfs"]
    xs = x / x.std(ddof=1)
    assert np.abs(got.sum(0) - xs).max() <= 1e-12 * np.abs(xs).max()
    a = _stats(got)
    b = _stats(orc.iceemdan(x, g["noise"], nimf, mi, nstd, solver=0))
    c = _stats(orc.iceemdan(x, g["noise"], nimf, mi, nstd, solver=1))
    for k in range(2):
        assert np.all(np.abs(a[k] - b[k]) <= 3.0 * np.maximum(np.abs(c[k] - b[k]), 0.01) + 1e-9)
