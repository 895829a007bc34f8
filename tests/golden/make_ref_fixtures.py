"""Generates the golden fixtures of the reference's own CUDA implementation (run on a GPU
machine after oracle/build_ref.sh has built oracle/_ref from the reference sources):

  ref_envelopes.npz   one envelope pass (the reference's kernels, CUB scans, cuSPARSE solves)
                      over seeded inputs (regenerated by the tests from ENV_CASES)
  ref_iceemdan.npz    one full iceemdanD decomposition and the N(0,1) noise it used (cuRAND
                      XORWOW seed 1234 on the device; the host generator differs in the last
                      bits, so the noise is stored)

Usage: python tests/golden/make_ref_fixtures.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

ENV_CASES = [(4, 1024, 7)]             # (nr, n, seed) of the envelope inputs
DEC_CASE = (32, 1024, 5, 50, 0.2)      # (nr, n, imfs, max_iter, nstd); signal two_tone_chirp


def envelope_input(nr, n, seed):
    rng = np.random.default_rng(seed)
    h = rng.standard_normal((nr, n))
    h[:, n // 2: n // 2 + 4] = 0.25  # a plateau
    return h


def device_normals(count, seed):
    """cuRAND CURAND_RNG_PSEUDO_DEFAULT normals generated on the device, as iceemdanD does."""
    import torch
    lib = ctypes.CDLL("libcurand.so.10")
    gen = ctypes.c_void_p()
    assert lib.curandCreateGenerator(ctypes.byref(gen), 100) == 0
    assert lib.curandSetPseudoRandomGeneratorSeed(gen, ctypes.c_ulonglong(seed)) == 0
    out = torch.empty(count + (count & 1), dtype=torch.float64, device="cuda:0")
    assert lib.curandGenerateNormalDouble(gen, ctypes.c_void_p(out.data_ptr()),
                                          ctypes.c_size_t(out.numel()), ctypes.c_double(0.0),
                                          ctypes.c_double(1.0)) == 0
    torch.cuda.synchronize()
    lib.curandDestroyGenerator(gen)
    return out[:count].cpu().numpy()


def main():
    import ref
    from __graft_entry__ import load_package
    load_package()
    from ceemdan_gpu_b200 import workloads
    out = {}
    for nr, n, seed in ENV_CASES:
        up, lo, cnt = ref.envelopes(envelope_input(nr, n, seed))
        out[f"up_{n}"], out[f"lo_{n}"], out[f"cnt_{n}"] = up, lo, cnt
    np.savez_compressed(os.path.join(HERE, "ref_envelopes.npz"), **out)
    nr, n, nimf, mi, nstd = DEC_CASE
    x = workloads.two_tone_chirp(n, seed=0)
    imfs, _ = ref.iceemdan(x, nr, nimf, mi, nstd)
    noise = device_normals(nr * n, 1234).reshape(nr, n)
    np.savez_compressed(os.path.join(HERE, "ref_iceemdan.npz"), imfs=imfs, noise=noise)
    print("fixtures written")


if __name__ == "__main__":
    main()
