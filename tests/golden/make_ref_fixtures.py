"""Generates the golden fixtures of the reference's own CUDA implementation (run on a GPU
machine after oracle/build_ref.sh has built oracle/_ref from the reference sources):

  ref_envelopes.npz   one envelope pass (the reference's kernels, CUB scans, cuSPARSE solves)
                      over seeded inputs (regenerated by the tests from ENV_CASES)
  ref_iceemdan.npz    one full iceemdanD decomposition and the N(0,1) noise it used (cuRAND
                      XORWOW seed 1234 on the device; the host generator differs in the last
                      bits, so the noise is stored), and the IMF statistics of a second run of
                      the same call: the reference's own run-to-run spread (its atomic sums
                      and cuSPARSE solves are not reproducible bit for bit)
  ref_knots.json      the knots of one envelope pass (the reference's extrema kernels, CUB
                      scans, compaction and end-knot rule) over seeded inputs up to the EEG
                      workload's length: per row and envelope the knot count and the SHA-256
                      of the positions (int32) and of the values (float64)

Usage: python tests/golden/make_ref_fixtures.py [output directory, default: this directory]
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
KNOT_CASES = [(4, 1024, 7), (3, 5003, 5), (2, 30001, 13), (1, 244032, 11)]  # knot inputs
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


def digest(a, dtype):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def imf_statistics(imfs):
    """Energy fraction and zero-crossing rate of each row (IMFs and residue)."""
    e = (imfs ** 2).sum(axis=1)
    zc = (np.diff(np.signbit(imfs).astype(np.int8), axis=1) != 0).mean(axis=1)
    return e / e.sum(), zc


def main():
    import json
    import ref
    from __graft_entry__ import load_package
    load_package()
    from ceemdan_gpu_b200 import workloads
    dest = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(dest, exist_ok=True)
    knots = {}
    for nr, n, seed in KNOT_CASES:
        kxM, kyM, kxm, kym, cnt = ref.knots(envelope_input(nr, n, seed))
        rows = []
        for r in range(nr):
            rows.append([{"count": int(cnt[e, r]),
                          "kx_sha256": digest(kx[r, :cnt[e, r]], "<i4"),
                          "ky_sha256": digest(ky[r, :cnt[e, r]], "<f8")}
                         for e, (kx, ky) in enumerate(((kxM, kyM), (kxm, kym)))])
        knots[f"{nr}x{n}_seed{seed}"] = rows
    with open(os.path.join(dest, "ref_knots.json"), "w") as f:
        json.dump(knots, f, indent=1)
    out = {}
    for nr, n, seed in ENV_CASES:
        up, lo, cnt = ref.envelopes(envelope_input(nr, n, seed))
        out[f"up_{n}"], out[f"lo_{n}"], out[f"cnt_{n}"] = up, lo, cnt
    np.savez_compressed(os.path.join(dest, "ref_envelopes.npz"), **out)
    nr, n, nimf, mi, nstd = DEC_CASE
    x = workloads.two_tone_chirp(n, seed=0)
    imfs, _ = ref.iceemdan(x, nr, nimf, mi, nstd)
    again, _ = ref.iceemdan(x, nr, nimf, mi, nstd)
    e2, z2 = imf_statistics(again)
    rel2 = np.abs(again - imfs).max(axis=1) / np.abs(imfs).max(axis=1)
    noise = device_normals(nr * n, 1234).reshape(nr, n)
    np.savez_compressed(os.path.join(dest, "ref_iceemdan.npz"), imfs=imfs, noise=noise,
                        run2_energy=e2, run2_zc=z2, run2_rel=rel2)
    print("fixtures written")


if __name__ == "__main__":
    main()
