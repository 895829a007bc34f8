"""End-to-end GPU parity at the EEG workload's length: whole decompositions of N = 244032
samples (17 IMFs, MaxIter 1000, noise sift cap 2000, Nstd 0.2) with a 4-realization ensemble,
bit for bit against the CPU oracle.

The oracle takes minutes at this length, so its results are stored as fingerprints
(tests/golden/oracle_eeg244032.json, made by tests/golden/make_oracle_fixtures.py): per-stage
lock-step iteration counts and the SHA-256 of the IMF array.  Both sides get the same external
white noise (numpy seed 1).  Cases: the synthetic EEG-shaped channel, and the reference's own
sample recording eegSampleDataCH1_244032.bin (raw float32) when present: copied into
oracle/_ref/data by oracle/build_ref.sh, or in the reference checkout (CEEMDAN_REFERENCE_DIR,
default: a sibling "reference" directory of the repository).
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _fixture():
    with open(os.path.join(HERE, "golden", "oracle_eeg244032.json")) as f:
        return json.load(f)


def _sha(a, dtype="<f8"):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def _input(name, wl):
    if name == "eeg_like_seed2":
        return wl.eeg_like(244032, seed=2)
    path = os.path.join(ROOT, "oracle", "_ref", "data", "eegSampleDataCH1_244032.bin")
    if not os.path.exists(path):
        ref_dir = os.environ.get("CEEMDAN_REFERENCE_DIR",
                                 os.path.join(os.path.dirname(ROOT), "reference"))
        path = os.path.join(ref_dir, "eegSampleDataCH1_244032.bin")
    if not os.path.exists(path):
        pytest.skip("the reference's sample recording is not present")
    return np.fromfile(path, dtype="<f4").astype(np.float64)


@pytest.mark.parametrize("name", ["eeg_like_seed2", "eegSampleDataCH1"])
def test_eeg_length_decomposition_bitexact(pkg, wl, cuda, name):
    import torch
    g = _fixture()
    case = g["cases"].get(name)
    if case is None:
        pytest.skip(f"{name}: no fixture")
    x = _input(name, wl)
    assert _sha(x) == case["input_sha256"]
    noise = torch.tensor(wl.white_noise(g["nr"], g["n"], 1), device=cuda)
    imfs, iters = pkg.iceemdan(torch.tensor(x, device=cuda), g["nr"], g["num_imfs"],
                               g["max_iter"], g["nstd"], noise=noise,
                               noise_sift_cap=g["noise_sift_cap"], return_iters=True)
    got = imfs.cpu().numpy()
    assert list(iters) == case["iters"]
    sub = np.array(case["subsample"])
    stride = case["subsample_stride"]
    err = np.abs(got[:, ::stride] - sub).max() / np.abs(sub).max()
    assert _sha(got) == case["sha256"], f"IMFs differ from the oracle (subsample rel {err:.3g})"


@pytest.mark.parametrize("name", ["eeg_like_seed2"])
def test_eeg_length_batched_bitexact(pkg, wl, cuda, name):
    """The same channel through the batched engine, next to a shorter channel: the batched
    loop runs the iteration counts and arithmetic of the oracle."""
    import torch
    g = _fixture()
    case = g["cases"][name]
    x = _input(name, wl)
    # the batched entry draws cuRAND noise; compare it with the plain engine on that noise
    ys = [torch.tensor(x, device=cuda), torch.tensor(wl.eeg_like(50000, seed=9), device=cuda)]
    outs, its = pkg.iceemdan_batched(ys, g["nr"], g["num_imfs"], g["max_iter"], g["nstd"],
                                     seed=3, noise_sift_cap=g["noise_sift_cap"],
                                     return_iters=True)
    for c, y in enumerate(ys):
        want, wit = pkg.iceemdan(y, g["nr"], g["num_imfs"], g["max_iter"], g["nstd"],
                                 seed=3 + c, noise_sift_cap=g["noise_sift_cap"],
                                 return_iters=True)
        assert its[c] == list(wit)
        assert torch.equal(outs[c], want)
