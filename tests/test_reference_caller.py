"""The reference's own sample driver, unmodified, relinked against libceemdan_b200.so.

sample_binary_file.cu (the reference's file-based example: reads a float32 EEG channel, calls
iceemdanS with NR = 200, 12 IMFs, MaxIter 300, Nstd 0.2, writes the modes) is compiled by
oracle/build_ref.sh from the reference checkout where it lies -- nothing is copied -- against
include/cudaICEEMDAN.cuh and linked with libceemdan_b200.so instead of the reference's
cudaICEEMDAN.cu / statistics.cu, into oracle/_ref together with the reference's sample
recording.  Its placeholder paths "/path/to/..." are redirected to a temporary directory by an
fopen shim (tests/path_shim.c, LD_PRELOAD).  The modes it writes must equal the tensor API's
iceemdanS result on the same recording bit for bit.  Skipped when oracle/_ref was built
without the reference sources.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_OUT = os.path.join(ROOT, "oracle", "_ref")  # built by oracle/build_ref.sh


@pytest.fixture(scope="module")
def sample_driver():
    exe = os.path.join(REF_OUT, "sample_binary_file")
    shim = os.path.join(REF_OUT, "path_shim.so")
    if not (os.path.exists(exe) and os.path.exists(shim)):
        pytest.skip("oracle/_ref has no relinked sample driver (needs the reference sources)")
    return exe, shim


def test_sample_driver_links_against_the_library_alone(sample_driver):
    exe, _ = sample_driver
    libs = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert "libceemdan_b200.so" in libs
    assert "cusparse" not in libs and "cublas" not in libs
    out = subprocess.run(["nm", "-D", "--undefined-only", exe], capture_output=True,
                         text=True, check=True).stdout
    assert "_Z9iceemdanSmmmmPiPfS0_f" in out


@pytest.mark.gpu
def test_sample_driver_modes_match_tensor_api(sample_driver, pkg, cuda, tmp_path):
    import torch
    exe, shim = sample_driver
    data = os.path.join(REF_OUT, "data", "eegSampleDataCH4.bin")
    if not os.path.exists(data):
        pytest.skip("eegSampleDataCH4.bin is not present")
    shutil.copy(data, tmp_path / "eegSampleDataCH4.bin")
    env = dict(os.environ, LD_PRELOAD=shim, CEEMDAN_PATH_DIR=str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Execution time" in r.stdout
    x = np.fromfile(data, dtype="<f4")
    n, nr, nimf, mi = x.size, 200, 12, 300  # the driver's configuration
    got = np.fromfile(tmp_path / "modes.bin", dtype="<f4").reshape(nimf, n)
    want = pkg.iceemdan(torch.tensor(x, device=cuda), nr, nimf, mi, 0.2, seed=1234)
    assert np.array_equal(got, want.cpu().numpy())
