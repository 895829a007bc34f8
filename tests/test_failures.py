"""Failure paths on the host side (no GPU fault is provoked): the host cancel word, an
allocation that cannot be satisfied, and the workspace going back to the library's memory
pool afterwards.  Each failing call must return its status without leaving device memory in
use and without poisoning the context for the next call."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _used(pkg):
    import torch
    torch.cuda.synchronize()
    return pkg.memory_stats()["used"]


def test_cancel_word_stops_plain_call(pkg, wl, cuda):
    import torch
    y = torch.tensor(wl.two_tone_chirp(4096, seed=1), device=cuda)
    pkg.iceemdan(y, 8, 5, 50, 0.2)  # the pool and module are set up
    before = _used(pkg)
    stop = ctypes.c_int32(1)
    with pytest.raises(pkg.CeemdanError) as ei:
        pkg.iceemdan(y, 8, 5, 50, 0.2, cancel=stop)
    assert ei.value.status == 6
    assert _used(pkg) == before
    # the next call runs normally and gives the usual result
    a = pkg.iceemdan(y, 8, 5, 50, 0.2)
    b = pkg.iceemdan(y, 8, 5, 50, 0.2, cancel=ctypes.c_int32(0))
    assert torch.equal(a, b)


def test_cancel_word_stops_batched_call(pkg, wl, cuda):
    import torch
    ys = [torch.tensor(wl.two_tone_chirp(n, seed=2), device=cuda) for n in (3000, 5000)]
    before = _used(pkg)
    with pytest.raises(pkg.CeemdanError) as ei:
        pkg.iceemdan_batched(ys, 6, 5, 50, 0.2, cancel=ctypes.c_int32(1))
    assert ei.value.status == 6
    assert _used(pkg) == before
    outs = pkg.iceemdan_batched(ys, 6, 5, 50, 0.2)
    for c, y in enumerate(ys):
        assert torch.equal(outs[c], pkg.iceemdan(y, 6, 5, 50, 0.2, seed=1234 + c))


def test_allocation_failure_returns_no_memory(pkg, cuda):
    """60000 realizations of 2^20 samples need about 500 GB per sift buffer: the first
    allocation fails, the call returns CEEMDAN_ERR_NO_MEMORY and frees what it held."""
    import torch
    n = 1 << 20
    y = torch.randn(n, dtype=torch.float64, device=cuda)
    before = _used(pkg)
    with pytest.raises(pkg.CeemdanError) as ei:
        pkg.iceemdan(y, 60000, 2, 1, 0.2)
    assert ei.value.status == 4
    assert _used(pkg) == before
    with pytest.raises(pkg.CeemdanError) as ei:
        pkg.iceemdan_batched([y, y], 60000, 2, 1, 0.2, wave_bytes=1)
    assert ei.value.status == 4
    assert _used(pkg) == before
    # the context is still usable
    small = torch.randn(2048, dtype=torch.float64, device=cuda)
    out = pkg.iceemdan(small, 4, 3, 10, 0.2)
    assert torch.isfinite(out).all()


def test_memory_stats_peak_covers_a_call(pkg, wl, cuda):
    import torch
    y = torch.tensor(wl.two_tone_chirp(8192, seed=3), device=cuda)
    pkg.memory_stats(reset_peak=True)
    pkg.iceemdan(y, 16, 5, 40, 0.2)
    torch.cuda.synchronize()
    st = pkg.memory_stats()
    # at least the sift state: h ping/pong, mean envelope, noise, noise modes (16 x 8192 each)
    assert st["peak"] >= (3 + 1 + 5) * 16 * 8192 * 8
    assert st["reserved"] >= st["peak"] >= st["used"]
