"""A reference-style C++ caller of iceemdanS / iceemdanD (tests/dropin_caller.cu) compiled
against include/cudaICEEMDAN.cuh and linked with libceemdan_b200.so alone: the relink a
reference caller does.  The build runs on CPU (nvcc cross-compiles); the GPU test runs it."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ceemdan-gpu_b200")


@pytest.fixture(scope="module")
def caller(built_lib, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("dropin") / "dropin_caller")
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-std=c++17", "-O2", os.path.join(ROOT, "tests", "dropin_caller.cu"),
                    "-I", os.path.join(ROOT, "include"), "-L", PKG, "-lceemdan_b200",
                    "-Xlinker", "-rpath", "-Xlinker", PKG, "-o", exe],
                   check=True, capture_output=True)
    return exe


def test_caller_links_against_the_drop_in_symbols(caller):
    out = subprocess.run(["nm", "-D", "--undefined-only", caller], capture_output=True,
                         text=True, check=True).stdout
    assert "_Z9iceemdanSmmmmPiPfS0_f" in out and "_Z9iceemdanDmmmmPiPdS0_d" in out
    libs = subprocess.run(["ldd", caller], capture_output=True, text=True).stdout
    assert "libceemdan_b200.so" in libs and "cusparse" not in libs


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f", "d"])
def test_caller_output_matches_tensor_api(caller, pkg, cuda, wl, tmp_path, dtype):
    import torch
    n, nr, nimf, mi = 2600, 8, 5, 60
    x = wl.eeg_like(n, seed=71).astype(np.float32 if dtype == "f" else np.float64)
    src, dst = tmp_path / "y.bin", tmp_path / "imfs.bin"
    x.tofile(src)
    r = subprocess.run([caller, str(src), str(dst), str(nr), str(nimf), str(mi), dtype],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.fromfile(dst, dtype=x.dtype).reshape(nimf, n)
    ref = pkg.iceemdan(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2, seed=1234).cpu().numpy()
    assert np.array_equal(got, ref)
