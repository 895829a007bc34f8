"""Generates tests/golden/oracle_eeg244032.json: fingerprints of CPU-oracle decompositions at
the EEG workload's length (N = 244032, 17 IMFs, MaxIter 1000, noise sift cap 2000, Nstd 0.2)
with a small ensemble (NR = 4, white noise from numpy seed 1, passed to both sides as external
noise), for the GPU end-to-end parity test (tests/test_parity_eeg.py).  The oracle takes
minutes at this length, so the test compares against these fingerprints instead of running it:
per-stage lock-step iteration counts, the SHA-256 of the IMF array's bytes (float64,
little-endian, row-major) and a strided subsample for diagnostics.

Cases: the synthetic EEG-shaped channel (workloads.eeg_like, seed 2) and, when the reference's
sample recording is present (eegSampleDataCH1_244032.bin, raw float32, in the directory named
by CEEMDAN_REFERENCE_DIR, default: a sibling "reference" directory of the repository), that
recording widened to float64.

    python tests/golden/make_oracle_fixtures.py
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

N, NR, NIMF, MAX_ITER, NSTD, CAP = 244032, 4, 17, 1000, 0.2, 2000
OUT = os.path.join(HERE, "oracle_eeg244032.json")


def reference_dir():
    return os.environ.get("CEEMDAN_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))


def inputs():
    from __graft_entry__ import load_package
    load_package()
    from ceemdan_gpu_b200 import workloads
    cases = {"eeg_like_seed2": workloads.eeg_like(N, seed=2)}
    path = os.path.join(reference_dir(), "eegSampleDataCH1_244032.bin")
    if os.path.exists(path):
        cases["eegSampleDataCH1"] = np.fromfile(path, dtype="<f4").astype(np.float64)
    noise = workloads.white_noise(NR, N, 1)
    return cases, noise


def fingerprint(imfs):
    return hashlib.sha256(np.ascontiguousarray(imfs, dtype="<f8").tobytes()).hexdigest()


def main():
    import oracle
    cases, noise = inputs()
    out = {"n": N, "nr": NR, "num_imfs": NIMF, "max_iter": MAX_ITER, "nstd": NSTD,
           "noise_sift_cap": CAP, "noise": "numpy default_rng(1).standard_normal((4, 244032))",
           "cases": {}}
    for name, x in cases.items():
        t0 = time.perf_counter()
        imfs, iters = oracle.iceemdan(x, noise, NIMF, MAX_ITER, NSTD, solver=1, chunk=16,
                                      noise_sift_cap=CAP, return_iters=True)
        dt = time.perf_counter() - t0
        out["cases"][name] = {"iters": [int(i) for i in iters], "sha256": fingerprint(imfs),
                              "input_sha256": fingerprint(x),
                              "subsample_stride": 997,
                              "subsample": imfs[:, ::997].tolist(),
                              "oracle_seconds": round(dt, 1)}
        print(name, "iterations", int(sum(iters)), f"{dt:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
