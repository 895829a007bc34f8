"""One channel's realizations split over ranks through the GPU engine
(ceemdan_plain_split_f64 / iceemdan_split), against one call holding every realization.

The ranks are processes with a gloo group on 127.0.0.1 that share this GPU: each runs its own
engine on its own realizations, and the exchanges (the lock-step stop flag of every sift
iteration, the ensemble sums passed along the ranks in realization order at the end of every
CEEMDAN stage) go through the host, so no kernel of one rank waits on another rank's kernels.
Every rank must return the one-call IMFs and iteration counts bit for bit, with external noise
(each rank its rows) and with cuRAND noise drawn for the whole ensemble.
"""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NR, N, NIMF, MAXIT, CAP = 7, 5000, 6, 80, 200


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, external):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        sys.path.insert(0, ROOT)
        from __graft_entry__ import load_package
        pkg = load_package()
        from ceemdan_gpu_b200 import multichannel, workloads
        dev = torch.device("cuda", 0)
        y = torch.tensor(workloads.eeg_like(N, seed=21), device=dev)
        r0, r1 = multichannel.realization_block(NR, rank, world)
        noise = None
        if external:
            noise = torch.tensor(workloads.white_noise(NR, N, 5)[r0:r1], device=dev)
        ens = multichannel.OrderedEnsemble(rank, world)
        imfs, iters = pkg.iceemdan_split(y, NR, r0, r1 - r0, NIMF, MAXIT, 0.2, ens, noise=noise,
                                         seed=31, noise_sift_cap=CAP, return_iters=True)
        np.savez(os.path.join(out_dir, f"part_{rank}.npz"), imfs=imfs.cpu().numpy(),
                 iters=np.array(iters))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,external", [(2, True), (3, True), (2, False)])
def test_engine_realization_split_equals_one_call(pkg, wl, cuda, tmp_path, world, external):
    import torch
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path), external), nprocs=world,
             join=True)
    y = torch.tensor(wl.eeg_like(N, seed=21), device=cuda)
    noise = torch.tensor(wl.white_noise(NR, N, 5), device=cuda) if external else None
    want, wit = pkg.iceemdan(y, NR, NIMF, MAXIT, 0.2, noise=noise, seed=31, noise_sift_cap=CAP,
                             return_iters=True)
    for r in range(world):
        got = np.load(os.path.join(tmp_path, f"part_{r}.npz"))
        assert list(got["iters"]) == list(wit)
        assert np.array_equal(got["imfs"], want.cpu().numpy())


def test_split_with_one_part_equals_plain_call(pkg, wl, cuda):
    """world = 1: the split entry with every realization is the plain call (its exchanges
    are identities), including the iteration-by-iteration stop test."""
    import torch
    from ceemdan_gpu_b200 import multichannel
    y = torch.tensor(wl.two_tone_chirp(3000, seed=2), device=cuda)
    got, git = pkg.iceemdan_split(y, 5, 0, 5, 5, 60, 0.2, multichannel.OrderedEnsemble(0, 1),
                                  seed=8, noise_sift_cap=120, return_iters=True)
    want, wit = pkg.iceemdan(y, 5, 5, 60, 0.2, seed=8, noise_sift_cap=120, return_iters=True)
    assert git == list(wit)
    assert torch.equal(got, want)
