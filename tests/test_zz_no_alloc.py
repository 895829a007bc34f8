"""The no-allocation tridiagonal entry point against the allocating one.

ceemdan_tridiag_noalloc_f64 exists for callers that cannot allocate device memory while they
run (real-time loops where an allocator call may synchronise the device, hosts that own all
device memory, framework plugins bound to the framework's memory pool); it works out of a
static scratch array in the library.  This file is collected last so that, if it fails, a
run that stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(batch, n, seed):
    rng = np.random.default_rng(seed)
    l = rng.uniform(1, 9, (batch, n))
    u = rng.uniform(1, 9, (batch, n))
    m = 2 * (l + u) + rng.uniform(0, 1, (batch, n))
    r = rng.standard_normal((batch, n))
    l[:, 0] = 0.0
    u[:, -1] = 0.0
    return l, m, u, r


@pytest.mark.parametrize("batch,n", [(3, 5000), (1, 150000), (20, 300)])
def test_noalloc_matches_allocating_solve_twice(pkg, cuda, batch, n):
    import torch
    L = pkg.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = None
    for call in range(2):
        l, m, u, r = (torch.tensor(a, device=cuda) for a in _systems(batch, n, 100 + call))
        want = torch.empty_like(r)
        got = torch.full_like(r, float("nan"))
        p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        assert L.ceemdan_tridiag_f64(batch, n, p(l), p(m), p(u), p(r), p(want), stream) == 0
        assert L.ceemdan_tridiag_noalloc_f64(batch, n, p(l), p(m), p(u), p(r), p(got),
                                             stream) == 0
        # the canonical solve is deterministic: the two entry points agree bit for bit
        assert torch.equal(got, want)
        if ref is not None:
            assert not torch.equal(got, ref)  # second call solved its own systems
        ref = got.clone()


def test_noalloc_rejects_oversized_requests(pkg, cuda):
    import torch
    L = pkg.lib()
    t = torch.zeros(8, device=cuda, dtype=torch.float64)
    p = ctypes.c_void_p(t.data_ptr())
    # 5*300000+64 doubles per system > the 1048576-double scratch: refused before launch
    assert L.ceemdan_tridiag_noalloc_f64(1, 300000, p, p, p, p, p, None) == 1
    assert b"static scratch" in L.ceemdan_last_error()


def test_noalloc_call_leaves_device_memory_unchanged(pkg, cuda):
    """After its first call on a device (which may load the library's device code and with it
    the static scratch), a call allocates nothing: the device's free memory is the same before
    and after it, and the library's memory pool is not touched."""
    import torch
    L = pkg.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    l, m, u, r = (torch.tensor(a, device=cuda) for a in _systems(4, 3000, 7))
    x = torch.empty_like(r)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    assert L.ceemdan_tridiag_noalloc_f64(4, 3000, p(l), p(m), p(u), p(r), p(x), stream) == 0
    pool0 = pkg.memory_stats()  # (creates the library's pool if this process had none)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert L.ceemdan_tridiag_noalloc_f64(4, 3000, p(l), p(m), p(u), p(r), p(x), stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    pool1 = pkg.memory_stats()
    assert free1 == free0
    assert pool1["used"] == pool0["used"] and pool1["reserved"] == pool0["reserved"]
