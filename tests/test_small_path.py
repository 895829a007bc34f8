"""The on-chip path for short rows (k_sift_small: one CTA per realization runs a whole stage,
with one bounded lock-step test per iteration) against the multi-kernel iteration.

Calls with N <= 8192 take the on-chip path (two CTAs per realization while 2·NR CTAs fit the
SMs, else one) (plain, timed and taped calls alike; a taped
stage records its tape slots from inside the kernel); the environment variable CEEMDAN_SMALL=0
sends them through the multi-kernel iteration, which the other parity tests pin to the CPU
oracle.  Both must give the same IMFs, iteration counts and gradients bit for bit.  The stop test's bounded wait is exercised without any fault: with a negative
spin limit the wait expects one arrival more than the launch has, every wait gives up, the
call returns CEEMDAN_ERR_TIMEOUT and the next call runs normally.
"""
import os

import pytest

pytestmark = pytest.mark.gpu


def _both(pkg, y, nr, nimf, mi, **kw):
    a = pkg.iceemdan(y, nr, nimf, mi, 0.2, return_iters=True, **kw)
    os.environ["CEEMDAN_SMALL"] = "0"
    try:
        b = pkg.iceemdan(y, nr, nimf, mi, 0.2, return_iters=True, **kw)
    finally:
        del os.environ["CEEMDAN_SMALL"]
    return a, b


@pytest.mark.parametrize("n,nr,nimf,mi,cap", [
    (4096, 50, 12, 300, 2000),   # config 1
    (8192, 16, 13, 100, 2000),   # a differentiation-workload signal's length
    (2049, 7, 8, 60, 300),       # one sample past a tile
    (100, 3, 4, 30, 100),        # one short tile
    (8192, 148, 6, 40, 80),      # one realization per SM
])
def test_small_path_equals_multi_kernel_iteration(pkg, wl, cuda, n, nr, nimf, mi, cap):
    import torch
    y = torch.tensor(wl.two_tone_chirp(n, seed=n % 97), device=cuda)
    (ia, ta), (ib, tb) = _both(pkg, y, nr, nimf, mi, seed=5, noise_sift_cap=cap)
    assert ta == tb
    assert torch.equal(ia, ib)


@pytest.mark.parametrize("checkpoint", [False, True])
def test_small_path_tape_equals_multi_kernel_tape(pkg, wl, cuda, checkpoint):
    """The taped forward on chip records the same tape (bitmaps, knot counts, end-rule flags,
    marks) as the multi-kernel iteration: the backward of both gives the same gradient."""
    import numpy as np
    import torch
    n, nr, nimf, mi = 3000, 6, 7, 60
    y = torch.tensor(wl.two_tone_chirp(n, seed=12), device=cuda)
    g = torch.tensor(np.random.default_rng(4).standard_normal((nimf, n)), device=cuda)

    def run():
        imfs, tape = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, seed=3, noise_sift_cap=150,
                                        checkpoint=checkpoint)
        gy = tape.backward(g)
        tape.free()
        return imfs, gy

    ia, ga = run()
    os.environ["CEEMDAN_SMALL"] = "0"
    try:
        ib, gb = run()
    finally:
        del os.environ["CEEMDAN_SMALL"]
    assert torch.equal(ia, ib)
    assert torch.equal(ga, gb)


def test_small_path_timed_call_reports_its_kernel(pkg, wl, cuda):
    """A call with per-kernel timing keeps the on-chip path and reports its time under
    sift_small (and nothing under the multi-kernel kinds)."""
    import torch
    y = torch.tensor(wl.two_tone_chirp(4096, seed=1), device=cuda)
    prof = {}
    a = pkg.iceemdan(y, 8, 6, 40, 0.2, profile=prof)
    assert prof["ms"]["sift_small"] > 0
    assert prof["ms"]["extrema"] == 0
    assert torch.equal(a, pkg.iceemdan(y, 8, 6, 40, 0.2))


def test_paired_ctas_equal_one_cta_per_realization(pkg, wl, cuda):
    """Two CTAs per realization (upper / lower envelope, handed over through L2) give the same
    result as one CTA doing both (CEEMDAN_SMALL_PAIR=0)."""
    import torch
    y = torch.tensor(wl.eeg_like(5000, seed=8), device=cuda)
    a, ia = pkg.iceemdan(y, 20, 8, 80, 0.2, seed=2, noise_sift_cap=200, return_iters=True)
    os.environ["CEEMDAN_SMALL_PAIR"] = "0"
    try:
        b, ib = pkg.iceemdan(y, 20, 8, 80, 0.2, seed=2, noise_sift_cap=200, return_iters=True)
    finally:
        del os.environ["CEEMDAN_SMALL_PAIR"]
    assert ia == ib
    assert torch.equal(a, b)


def test_small_path_with_external_noise_matches_oracle(pkg, orc, wl, cuda):
    import torch
    n, nr, nimf, mi = 3000, 6, 7, 80
    x = wl.eeg_like(n, seed=4)
    noise = wl.white_noise(nr, n, 9)
    got, it = pkg.iceemdan(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2,
                           noise=torch.tensor(noise, device=cuda), noise_sift_cap=200,
                           return_iters=True)
    want, wit = orc.iceemdan(x, noise, nimf, mi, 0.2, solver=1, chunk=16, noise_sift_cap=200,
                             return_iters=True)
    assert list(it) == list(wit)
    assert (got.cpu().numpy() == want).all()


def test_stop_test_wait_gives_up_with_timeout_status(pkg, wl, cuda):
    import torch
    y = torch.tensor(wl.two_tone_chirp(2048, seed=3), device=cuda)
    with pytest.raises(pkg.CeemdanError) as ei:
        pkg.iceemdan(y, 8, 5, 30, 0.2, spin_limit=-1000)
    assert ei.value.status == 5
    # the context is usable and the next call gives the usual result
    a = pkg.iceemdan(y, 8, 5, 30, 0.2)
    os.environ["CEEMDAN_SMALL"] = "0"
    try:
        b = pkg.iceemdan(y, 8, 5, 30, 0.2)
    finally:
        del os.environ["CEEMDAN_SMALL"]
    assert torch.equal(a, b)
