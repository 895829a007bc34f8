"""The batched engine (ceemdan_batched_f64) against the one-channel engine.

Every channel of a batch must come out bit for bit as ceemdan_plain_f64 of that channel with
the same seed (seed + channel index): the batched loop runs the same kernels and the same
stage arithmetic, only driven from the device, with channels at different stages at the same
time.  The one-channel engine is itself pinned bit-exact to the CPU oracle
(test_gpu_parity.py), and one small batch is checked against the oracle directly.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


def _channels(wl, lengths, seed0=50):
    return [wl.two_tone_chirp(n, seed=seed0 + i) if i % 2 == 0 else
            wl.eeg_like(n, seed=seed0 + i) for i, n in enumerate(lengths)]


def _plain(pkg, y, nr, nimf, max_iter, seed, cap):
    return pkg.iceemdan(y, nr, nimf, max_iter, 0.2, seed=seed, noise_sift_cap=cap,
                        return_iters=True)


@pytest.mark.parametrize("lengths,nr,nimf,max_iter,cap", [
    ([5000, 3001, 8192, 2053, 700], 8, 6, 100, 300),   # ragged, odd lengths, tile edges
    ([4096], 16, 8, 60, 200),                          # one channel
    ([1024, 1024, 1024], 4, 5, 40, 80),                # equal lengths, different seeds
])
def test_batched_equals_plain_per_channel(pkg, wl, cuda, lengths, nr, nimf, max_iter, cap):
    import torch
    xs = _channels(wl, lengths)
    ys = [torch.tensor(x, device=cuda) for x in xs]
    prof = {}
    outs, iters = pkg.iceemdan_batched(ys, nr, nimf, max_iter, 0.2, seed=77,
                                       noise_sift_cap=cap, return_iters=True, profile=prof)
    for c, y in enumerate(ys):
        want, wit = _plain(pkg, y, nr, nimf, max_iter, 77 + c, cap)
        assert iters[c] == list(wit), f"channel {c}: iteration counts differ"
        assert torch.equal(outs[c], want), f"channel {c}: IMFs differ"
    assert prof["counters"]["waves"] == 1
    assert prof["counters"]["launches"] > 0


def test_batched_waves_and_graph_depths_agree(pkg, wl, cuda):
    """Waves (a small memory budget forces one channel per wave) and other graph depths give
    the same results as one wave."""
    import torch
    xs = _channels(wl, [3000, 6000, 2500], seed0=90)
    ys = [torch.tensor(x, device=cuda) for x in xs]
    ref = pkg.iceemdan_batched(ys, 6, 6, 80, 0.2, seed=5, noise_sift_cap=150)
    prof = {}
    waves = pkg.iceemdan_batched(ys, 6, 6, 80, 0.2, seed=5, noise_sift_cap=150,
                                 wave_bytes=1, profile=prof)
    assert prof["counters"]["waves"] == 3
    deep = pkg.iceemdan_batched(ys, 6, 6, 80, 0.2, seed=5, noise_sift_cap=150, group=3)
    for a, b, c in zip(ref, waves, deep):
        assert torch.equal(a, b)
        assert torch.equal(a, c)


def test_batched_against_oracle(pkg, orc, wl, cuda):
    """One ragged batch against the CPU oracle directly, fed the same cuRAND noise (device
    generator, seed 11 + channel)."""
    from test_gpu_parity import _curand_device_normals
    import torch
    lengths = [2100, 1500, 777]
    xs = _channels(wl, lengths, seed0=7)
    ys = [torch.tensor(x, device=cuda) for x in xs]
    nr, nimf, mi, cap = 4, 5, 50, 120
    outs, iters = pkg.iceemdan_batched(ys, nr, nimf, mi, 0.2, seed=11, noise_sift_cap=cap,
                                       return_iters=True)
    for c, x in enumerate(xs):
        n = lengths[c]
        noise = _curand_device_normals(nr * n, 11 + c, cuda).reshape(nr, n).cpu().numpy()
        want, wit = orc.iceemdan(x, noise, nimf, mi, 0.2, solver=1, chunk=16,
                                 noise_sift_cap=cap, return_iters=True)
        assert list(iters[c]) == list(wit)
        assert np.array_equal(outs[c].cpu().numpy(), want)
