"""The C-ABI library builds, loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_c_symbols():
    src = open(os.path.join(ROOT, "include", "ceemdan_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(ceemdan_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol(built_lib, pkg):
    syms = _declared_c_symbols()
    assert "ceemdan_plain_f64" in syms and len(syms) >= 9
    L = ctypes.CDLL(built_lib)
    for s in syms:
        assert hasattr(L, s), s
    # the C++-linkage drop-in of cudaICEEMDAN.cuh:26
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True,
                         text=True, check=True).stdout
    assert "_Z9iceemdanDmmmmPiPdS0_d" in out
    assert set(pkg.EXPORTS) == set(syms)


def test_library_is_sm100a_only(built_lib):
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", built_lib],
                         capture_output=True, text=True).stdout
    assert "sm_100a" in out
    assert not re.search(r"sm_(?!100a)\d+", out.replace("sm_100a", ""))


def test_build_info_and_status_strings(pkg, built_lib):
    L = pkg.lib()
    assert b"sm_100a" in L.ceemdan_build_info()
    for code in range(7):
        assert L.ceemdan_status_string(code)
    o = pkg.default_options()
    assert o.noise_sift_cap == 2000 and o.seed == 1234 and o.sd == 0.05 and o.sd2 == 0.5


def test_invalid_arguments_rejected_before_gpu_work(pkg, built_lib):
    L = pkg.lib()
    # n < 4 / num_imfs < 2 / nr == 0 are rejected on the host: no device is touched
    assert L.ceemdan_plain_f64(4, 3, 5, 10, None, None, None, 0.2, None, None) == 1
    assert L.ceemdan_plain_f64(0, 100, 5, 10, None, None, None, 0.2, None, None) == 1
    assert L.ceemdan_plain_f64(4, 100, 1, 10, None, None, None, 0.2, None, None) == 1
    bad = pkg.default_options()
    bad.struct_size = 3
    assert L.ceemdan_plain_f64(4, 100, 5, 10, 1, 1, 1, 0.2, ctypes.byref(bad), None) == 1
