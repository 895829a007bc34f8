"""Multi-rank host logic on CPU: two gloo ranks shard ragged channels, decompose their share
(with the CPU oracle standing in for the GPU engine), gather to rank 0, and reduce the timing
with max over ranks and the work units with a sum.  No GPU and no NCCL: the same code paths
run over NCCL on GPUs."""
import importlib.util
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _multichannel():
    spec = importlib.util.spec_from_file_location(
        "multichannel", os.path.join(ROOT, "ceemdan-gpu_b200", "multichannel.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _channels():
    rng = np.random.default_rng(7)
    lengths = [300, 520, 260, 410, 333, 600]
    return [np.cumsum(rng.standard_normal(n)) * 0.1 + rng.standard_normal(n) for n in lengths]


NR, NIMF, MAXIT = 4, 4, 40


def _decompose(ch):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    noise = np.random.default_rng(len(ch)).standard_normal((NR, len(ch)))
    return oracle.iceemdan(ch, noise, NIMF, MAXIT, 0.2, solver=1, noise_sift_cap=60)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mc = _multichannel()
        res = mc.decompose_channels(_channels(), _decompose, rank=rank, world=world)
        # timing reduction: every rank must see the slowest rank's time
        mx = mc.max_over_ranks(10.0 + rank, world)
        # work units of ranks whose shares differ add up
        sm = mc.sum_over_ranks(1.5 + rank, world)
        np.save(os.path.join(out_dir, f"max_{rank}.npy"), np.array([mx, sm]))
        if rank == 0:
            np.savez(os.path.join(out_dir, "gathered.npz"), **{str(k): v for k, v in res.items()})
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_partitions_and_balances():
    mc = _multichannel()
    lengths = [250_000, 30_000, 120_000, 240_000, 90_000, 60_000, 200_000, 35_000]
    for world in (1, 2, 3, 4, 8):
        parts = mc.shard(lengths, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(lengths)))
        loads = [sum(lengths[i] for i in p) for p in parts]
        # longest-first greedy: no rank exceeds the average by more than the longest channel
        assert max(loads) <= sum(lengths) / world + max(lengths)
        assert parts == mc.shard(lengths, world)  # deterministic
        for r in range(world):
            assert mc.rank_channels(lengths, r, world) == parts[r]
    with pytest.raises(ValueError):
        mc.shard(lengths, 0)


def test_two_gloo_ranks_shard_decompose_gather(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    gathered = np.load(tmp_path / "gathered.npz")
    chans = _channels()
    assert sorted(int(k) for k in gathered.files) == list(range(len(chans)))
    for i, ch in enumerate(chans):
        assert np.array_equal(gathered[str(i)], _decompose(ch))
    for r in range(world):
        mx, sm = np.load(tmp_path / f"max_{r}.npy")
        assert (float(mx), float(sm)) == (11.0, 4.0)


def test_single_rank_needs_no_process_group():
    mc = _multichannel()
    res = mc.decompose_channels(_channels()[:2], lambda c: len(c), rank=0, world=1)
    assert res == {0: 300, 1: 520}
    assert mc.max_over_ranks(3.5, 1) == 3.5
    assert mc.sum_over_ranks(3.5, 1) == 3.5


@pytest.mark.gpu
def test_streams_batch_equals_single_calls(pkg, cuda, wl):
    """Ragged channels decomposed side by side on one GPU (3 streams) equal the one-at-a-time
    results bit for bit, and the side-by-side run is timed against the sequential one."""
    import time
    import torch
    mc = _multichannel()
    lengths = [9000, 3000, 14000, 5000, 11000, 4096]
    chans = [wl.eeg_like(n, seed=20 + i) for i, n in enumerate(lengths)]
    kw = dict(noise_sift_cap=150)
    torch.cuda.synchronize()
    t0 = time.time()
    seq = [pkg.iceemdan(torch.tensor(c, device=cuda), 24, 6, 60, 0.2, seed=1234 + i, **kw)
           for i, c in enumerate(chans)]
    torch.cuda.synchronize()
    t1 = time.time()
    par = mc.decompose_on_streams(pkg, chans, 24, 6, 60, 0.2, streams=3, device=cuda, **kw)
    torch.cuda.synchronize()
    t2 = time.time()
    print(f"sequential {t1 - t0:.3f}s, 3 streams {t2 - t1:.3f}s")
    for a, b in zip(seq, par):
        assert torch.equal(a, b)


def _gradient(ch):
    """d/dy of sum_k w_k |IMF_k|^2 for one signal (oracle taped forward + vjp)."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    noise = np.random.default_rng(len(ch)).standard_normal((NR, len(ch)))
    t = oracle.Tape(ch, noise, NIMF, MAXIT, 0.2, solver=1, noise_sift_cap=60)
    w = np.random.default_rng(4).uniform(size=NIMF)
    return t.vjp(2.0 * w[:, None] * t.imfs)


def _worker_grad(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = _multichannel().decompose_channels(_channels(), _gradient, rank=rank, world=world)
        if rank == 0:
            np.savez(os.path.join(out_dir, "grads.npz"), **{str(k): v for k, v in res.items()})
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_gradients(tmp_path):
    """The differentiation form shards like the decomposition: independent signals, no
    collective on the data path, gradients gathered to rank 0."""
    import torch.multiprocessing as mp
    mp.start_processes(_worker_grad, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    grads = np.load(tmp_path / "grads.npz")
    chans = _channels()
    assert sorted(int(k) for k in grads.files) == list(range(len(chans)))
    for i, ch in enumerate(chans):
        assert np.array_equal(grads[str(i)], _gradient(ch))


SPLIT_NR, SPLIT_N, SPLIT_IMF, SPLIT_MAXIT = 7, 1500, 5, 60


def _split_worker(rank, world, port, out_dir):
    import sys
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        mc = _multichannel()
        x = np.sin(np.arange(SPLIT_N) * 0.05) + np.random.default_rng(3).standard_normal(SPLIT_N)
        noise = np.random.default_rng(11).standard_normal((SPLIT_NR, SPLIT_N))
        r0, r1 = mc.realization_block(SPLIT_NR, rank, world)
        ops = mc.OrderedEnsemble(rank, world)
        imfs, iters = oracle.iceemdan_split(x, noise[r0:r1], SPLIT_NR, rank, world, ops,
                                            SPLIT_IMF, SPLIT_MAXIT, 0.2, noise_sift_cap=150,
                                            threads=1, return_iters=True)
        np.savez(os.path.join(out_dir, f"split_{rank}.npz"), imfs=imfs, iters=iters)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_realization_split_equals_one_rank(tmp_path, world):
    """One channel's realizations split over gloo ranks (the oracle standing in for the engine):
    the lock-step stop test reduced over the ranks and the ensemble sums continued across them
    in realization order give every rank the one-rank decomposition bit for bit."""
    import sys
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    port = _free_port()
    mp.spawn(_split_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    x = np.sin(np.arange(SPLIT_N) * 0.05) + np.random.default_rng(3).standard_normal(SPLIT_N)
    noise = np.random.default_rng(11).standard_normal((SPLIT_NR, SPLIT_N))
    want, wit = oracle.iceemdan(x, noise, SPLIT_IMF, SPLIT_MAXIT, 0.2, solver=1,
                                noise_sift_cap=150, return_iters=True)
    for r in range(world):
        got = np.load(os.path.join(tmp_path, f"split_{r}.npz"))
        assert np.array_equal(got["iters"], wit)
        assert np.array_equal(got["imfs"], want)


def test_realization_blocks_cover_in_order():
    mc = _multichannel()
    for nr in (1, 7, 100, 1000):
        for world in (1, 2, 3, 8):
            blocks = [mc.realization_block(nr, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == nr
            for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
                assert a1 == b0
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
