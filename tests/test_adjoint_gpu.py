"""The backward entry (ceemdan_forward_taped_f64 + ceemdan_backward_f64) against the CPU
oracle's reverse pass, which tests/test_adjoint_oracle.py pins with central differences.

The GPU tests compare gradients of the weighted-energy loss sum_k w_k |IMF_k|^2 (w_k ~ U(0, 1),
seed 4) on the same seeded inputs and noise; the CPU tests check the entry points' argument
handling without touching a device."""
import ctypes

import numpy as np
import pytest


def _weights(nimf):
    return np.random.default_rng(4).uniform(size=nimf)


def test_backward_entry_rejects_bad_arguments_on_the_host(pkg, built_lib):
    L = pkg.lib()
    assert L.ceemdan_backward_f64(None, None, None, None) == 1
    assert L.ceemdan_tape_bytes(None) == 0
    assert L.ceemdan_tape_iterations(None, 0) == -1
    L.ceemdan_tape_free(None)
    h = ctypes.c_void_p()
    # no tape_out; more realizations than the reverse pass launches
    assert L.ceemdan_forward_taped_f64(4, 100, 5, 10, None, None, None, 0.2, None, None,
                                       None) == 1
    assert L.ceemdan_forward_taped_f64(40000, 100, 5, 10, None, None, None, 0.2, None, None,
                                       ctypes.byref(h)) == 1
    assert not h


def test_tape_slot_layout(tmp_path):
    """The tape slot layout the recording and reverse-pass kernels index with (host check,
    compiled from the library's own header)."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "tape_layout_check"
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O1",
                    os.path.join(root, "tests", "tape_layout_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0" in out.stdout


def _run(pkg, orc, wl, cuda, n, nr, nimf, mi, cap, seed=0, signal="chirp"):
    import torch
    x = wl.two_tone_chirp(n, seed=seed) if signal == "chirp" else wl.eeg_like(n, seed=seed)
    noise = wl.white_noise(nr, n, 1)
    imfs, tape = pkg.iceemdan_taped(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2,
                                    noise=torch.tensor(noise, device=cuda), noise_sift_cap=cap)
    t = orc.Tape(x, noise, nimf, mi, 0.2, solver=1, chunk=16, noise_sift_cap=cap)
    return x, imfs, tape, t


@pytest.mark.gpu
def test_taped_forward_is_the_plain_forward(pkg, orc, wl, cuda):
    import torch
    n, nr, nimf, mi, cap = 4096, 16, 12, 300, 600
    x, imfs, tape, t = _run(pkg, orc, wl, cuda, n, nr, nimf, mi, cap)
    plain = pkg.iceemdan(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2,
                         noise=torch.tensor(wl.white_noise(nr, n, 1), device=cuda),
                         noise_sift_cap=cap)
    assert torch.equal(imfs, plain)
    assert np.array_equal(imfs.cpu().numpy(), t.imfs)
    assert tape.iterations == t.iterations()
    assert tape.bytes > 0


def _check_vjp(tape, t, imfs, nimf):
    """The backward performs the oracle's vjp operations in the oracle's order: the gradients
    are identical bit for bit (the oracle's vjp is pinned by central differences)."""
    import torch
    w = _weights(nimf)
    g = 2.0 * torch.tensor(w, device=imfs.device)[:, None] * imfs
    gy = tape.backward(g).cpu().numpy()
    ref = t.vjp(2.0 * w[:, None] * t.imfs)
    err = np.abs(gy - ref).max() / np.abs(ref).max()
    assert np.array_equal(gy, ref), f"backward differs from the oracle's vjp (rel {err:.3g})"
    return gy, ref


@pytest.mark.gpu
@pytest.mark.parametrize("n,nr,nimf,mi,cap", [
    (2048, 8, 8, 100, 200),      # dense and sparse stages, one partition level
    (5000, 6, 9, 60, 150),       # ragged length, knots across three tiles
])
def test_backward_matches_oracle_vjp(pkg, orc, wl, cuda, n, nr, nimf, mi, cap):
    _, imfs, tape, t = _run(pkg, orc, wl, cuda, n, nr, nimf, mi, cap)
    _check_vjp(tape, t, imfs, nimf)


@pytest.mark.gpu
def test_backward_differentiation_workload_signal(pkg, orc, wl, cuda):
    """One signal of the differentiation workload: N=8192 as the two-tone chirp recipe (seed
    10), NR=50, MaxIter=100, 13 IMFs, reference noise cap 2000."""
    _, imfs, tape, t = _run(pkg, orc, wl, cuda, 8192, 50, 13, 100, 2000, seed=10)
    _check_vjp(tape, t, imfs, 13)


@pytest.mark.gpu
def test_backward_through_stale_means_caps_and_end_rules(pkg, orc, wl, cuda):
    """Short signal (stale mean envelopes, splines too short for the end rule) and a sift cap
    of 3 (every realization exports its mode at the cap)."""
    _, imfs, tape, t = _run(pkg, orc, wl, cuda, 40, 3, 5, 3, 50, seed=7)
    _check_vjp(tape, t, imfs, 5)


@pytest.mark.gpu
def test_autograd_function_gives_the_backward_entry(pkg, orc, wl, cuda):
    import torch
    n, nr, nimf, mi, cap = 3000, 6, 8, 80, 200
    x = wl.eeg_like(n, seed=11)
    noise = torch.tensor(wl.white_noise(nr, n, 1), device=cuda)
    y = torch.tensor(x, device=cuda, requires_grad=True)
    imfs = pkg.iceemdan_autograd(y, nr, nimf, mi, 0.2, noise=noise, noise_sift_cap=cap)
    w = torch.tensor(_weights(nimf), device=cuda)
    loss = (w[:, None] * imfs ** 2).sum()
    loss.backward()
    t = orc.Tape(x, noise.cpu().numpy(), nimf, mi, 0.2, solver=1, noise_sift_cap=cap)
    ref = t.vjp(2.0 * _weights(nimf)[:, None] * t.imfs)
    assert np.array_equal(y.grad.cpu().numpy(), ref)


@pytest.mark.gpu
def test_gradients_on_streams_equal_single_calls(pkg, wl, cuda):
    """Signals of one length on several streams, sharing the noise phase: every gradient
    equals the one of a single taped forward + backward."""
    import torch
    from ceemdan_gpu_b200 import multichannel
    n, nr, nimf, mi, cap = 2048, 8, 7, 60, 150
    ys = [torch.tensor(wl.two_tone_chirp(n, seed=20 + s), device=cuda) for s in range(5)]
    w = torch.tensor(_weights(nimf), device=cuda)
    _, state = pkg.iceemdan(ys[0], nr, nimf, mi, 0.2, seed=1, noise_sift_cap=cap,
                            return_noise_state=True)
    got = multichannel.gradients_on_streams(pkg, ys, nr, nimf, mi, 0.2,
                                            lambda imfs: 2.0 * w[:, None] * imfs, streams=3,
                                            device=cuda, seed=1, noise_state=state,
                                            noise_sift_cap=cap)
    for y, g in zip(ys, got):
        imfs, tape = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, seed=1, noise_sift_cap=cap)
        assert torch.equal(g, tape.backward(2.0 * w[:, None] * imfs))


@pytest.mark.gpu
def test_checkpointed_backward_equals_full_tape(pkg, orc, wl, cuda):
    """Checkpoint and recompute: per-stage checkpoints instead of every iteration, the backward
    re-runs each stage; gradients equal the full tape's and the oracle's bit for bit, and the
    tape's size does not depend on the iteration counts (checkpoints pay off when stages run
    more than about 64 iterations on average, as the long signal stages of the EEG workload
    do; these short test stages do not)."""
    import torch
    n, nr, nimf, mi, cap = 2048, 8, 6, 300, 300
    x = wl.two_tone_chirp(n, seed=5)
    noise = torch.tensor(wl.white_noise(nr, n, 1), device=cuda)
    y = torch.tensor(x, device=cuda)
    w = torch.tensor(_weights(nimf), device=cuda)
    imfs_f, full = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, noise=noise, noise_sift_cap=cap)
    imfs_c, ckpt = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, noise=noise, noise_sift_cap=cap,
                                      checkpoint=True)
    assert torch.equal(imfs_f, imfs_c)
    assert ckpt.iterations == full.iterations
    # noise modes, stage inputs and statistics, then per stage h0, mean envelope, fraction
    assert ckpt.bytes == 8 * (nimf * nr * n + (nimf - 1) * n + 2 * (nimf - 1) +
                              (nimf - 1) * (2 * nr * n + nr))
    g = 2.0 * w[:, None] * imfs_f
    gc = ckpt.backward(g)
    assert torch.equal(gc, full.backward(g))
    assert torch.equal(gc, ckpt.backward(g))  # the checkpoints survive a backward
    t = orc.Tape(x, noise.cpu().numpy(), nimf, mi, 0.2, solver=1, noise_sift_cap=cap)
    assert np.array_equal(gc.cpu().numpy(), t.vjp(2.0 * _weights(nimf)[:, None] * t.imfs))


@pytest.mark.gpu
@pytest.mark.parametrize("n,block", [(2048, 3), (9000, 2), (9000, 4)])
def test_checkpointed_backward_in_realization_blocks(pkg, wl, cuda, n, block):
    """A checkpointed backward re-runs and reverses the realizations a block at a time (each
    block for the stage's recorded iteration count, so a block whose realizations all finish
    early still runs as long as the whole ensemble did); any block size gives the full tape's
    gradient bit for bit: blocks of 3 of 7 on the on-chip path, blocks of 2 and of 4 (a
    shorter last block) of 7 on the multi-kernel path."""
    import os
    import torch
    nr, nimf, mi, cap = 7, 5, 120, 150
    y = torch.tensor(wl.eeg_like(n, seed=6), device=cuda)
    w = torch.tensor(_weights(nimf), device=cuda)
    imfs, full = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, seed=4, noise_sift_cap=cap)
    _, ckpt = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, seed=4, noise_sift_cap=cap,
                                 checkpoint=True)
    g = 2.0 * w[:, None] * imfs
    want = full.backward(g)
    os.environ["CEEMDAN_BACKWARD_BLOCK"] = str(block)
    try:
        got = ckpt.backward(g)
    finally:
        del os.environ["CEEMDAN_BACKWARD_BLOCK"]
    assert torch.equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [3000, 9000])
def test_level_by_level_transposed_solve_equals_cta_solve(pkg, wl, cuda, n):
    """The backward's transposed spline solves level by level over the whole grid
    (psolve_launch, the default for long splines) give the one-CTA-per-spline solve's
    gradient bit for bit (CEEMDAN_ADJ_SOLVE forces either)."""
    import os
    import torch
    nr, nimf, mi, cap = 6, 5, 100, 150
    y = torch.tensor(wl.eeg_like(n, seed=9), device=cuda)
    w = torch.tensor(_weights(nimf), device=cuda)
    imfs, tape = pkg.iceemdan_taped(y, nr, nimf, mi, 0.2, seed=12, noise_sift_cap=cap)
    g = 2.0 * w[:, None] * imfs
    got = {}
    for mode in ("cta", "grid"):
        os.environ["CEEMDAN_ADJ_SOLVE"] = mode
        try:
            got[mode] = tape.backward(g)
        finally:
            del os.environ["CEEMDAN_ADJ_SOLVE"]
    assert torch.equal(got["cta"], got["grid"])
