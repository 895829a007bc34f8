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
    # the C++-linkage drop-ins of cudaICEEMDAN.cuh:25-26
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True,
                         text=True, check=True).stdout
    assert "_Z9iceemdanDmmmmPiPdS0_d" in out
    assert "_Z9iceemdanSmmmmPiPfS0_f" in out
    assert set(pkg.DROPIN_SYMBOLS.values()) <= set(out.split())
    assert set(pkg.EXPORTS) == set(syms)


def test_library_is_sm100a_only(built_lib):
    """Every kernel entry ptxas compiled for the library (its -v log, one file per source)
    targets sm_100a and nothing else; the Makefile passes a single -gencode."""
    build = os.path.join(ROOT, "ceemdan-gpu_b200", "_build")
    if not os.path.isdir(build):
        subprocess.run(["make", "-C", os.path.join(ROOT, "ceemdan-gpu_b200")], check=True,
                       capture_output=True)
    targets = []
    for f in sorted(os.listdir(build)):
        if f.endswith(".ptxas.txt"):
            targets += re.findall(r"Compiling entry function '[^']+' for '(\w+)'",
                                  open(os.path.join(build, f)).read())
    assert targets and set(targets) == {"sm_100a"}
    mk = open(os.path.join(ROOT, "ceemdan-gpu_b200", "Makefile")).read()
    assert re.findall(r"-gencode\s+arch=(\S+)", mk) == ["compute_100a,code=sm_100a"]


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


def test_batch_rejects_invalid_arguments_before_gpu_work(pkg, built_lib):
    L = pkg.lib()
    lengths = (ctypes.c_size_t * 2)(100, 3)
    ptrs = (ctypes.c_void_p * 2)(1, 1)
    assert L.ceemdan_batch_f64(0, lengths, ptrs, ptrs, 4, 5, 10, 0.2, None, 2) == 1
    assert L.ceemdan_batch_f64(2, lengths, ptrs, ptrs, 4, 5, 10, 0.2, None, 2) == 1  # n < 4
    assert b"channel 1" in L.ceemdan_last_error()
    lengths[1] = 100
    assert L.ceemdan_batch_f64(2, lengths, ptrs, ptrs, 4, 5, 10, 0.2, None, 0) == 1  # streams
    o = pkg.default_options()
    o.d_noise = 1  # external noise has no per-channel meaning here
    assert L.ceemdan_batch_f64(2, lengths, ptrs, ptrs, 4, 5, 10, 0.2, ctypes.byref(o), 2) == 1


def test_split_rejects_invalid_arguments_before_gpu_work(pkg, built_lib):
    """ceemdan_plain_split_f64: a missing split, missing exchanges, a rank outside the group,
    a block past the ensemble or a tape-free call with noise-state buffers are rejected on the
    host, before any device work."""
    L = pkg.lib()
    ok = pkg._ALL_FINISHED(lambda c, local: local)
    xch = pkg._EXCHANGE(lambda c, p, n: 0)

    def split(**kw):
        sp = pkg.Split()
        sp.nr_total, sp.first, sp.rank, sp.world = 8, 0, 0, 2
        sp.all_finished, sp.recv_partial, sp.send_partial, sp.broadcast_last = ok, xch, xch, xch
        for k, v in kw.items():
            setattr(sp, k, v)
        return sp

    def call(sp, nr=4, opt=None):
        return L.ceemdan_plain_split_f64(nr, 100, 5, 10, 1, 1, 1, 0.2,
                                         ctypes.byref(opt) if opt else None,
                                         ctypes.byref(sp) if sp is not None else None, None)

    assert call(None) == 1
    assert call(split(rank=2)) == 1                 # rank outside 0..world-1
    assert call(split(first=6)) == 1                # 6 + 4 realizations past nr_total = 8
    assert call(split(world=0)) == 1
    assert call(split(all_finished=pkg._ALL_FINISHED())) == 1  # missing exchange
    o = pkg.default_options()
    o.d_noise_state_out = 1                          # the split takes no noise state
    assert call(split(), opt=o) == 1
    assert b"split" in L.ceemdan_last_error()


def test_tensor_entry_points_reject_host_tensors(pkg, built_lib):
    """The tensor entry points take CUDA tensors only: a host tensor (or a wrong dtype or
    shape) raises CeemdanError with status 1 before anything runs; there is no CPU path."""
    import pytest
    import torch
    y = torch.zeros(1000, dtype=torch.float64)
    calls = [
        lambda: pkg.iceemdan(y, 4, 3, 50, 0.2),
        lambda: pkg.iceemdan(y.float(), 4, 3, 50, 0.2),
        lambda: pkg.iceemdan(y.view(10, 100), 4, 3, 50, 0.2),
        lambda: pkg.iceemdan_batch([y, y[:800]], 4, 3, 50, 0.2),
        lambda: pkg.iceemdan_batched([y, y[:800]], 4, 3, 50, 0.2),
        lambda: pkg.iceemdan_split(y, 4, 0, 2, 3, 50, 0.2, None),
        lambda: pkg.iceemdan_taped(y, 4, 3, 50, 0.2),
    ]
    for call in calls:
        with pytest.raises(pkg.CeemdanError) as e:
            call()
        assert e.value.status == 1 and "CUDA tensor" in str(e.value)


def test_options_struct_matches_c_layout(pkg, built_lib):
    """ceemdan_default_options writes sizeof(ceemdan_options) into struct_size: the ctypes
    mirror must have the same size (fields appended at the end keep old callers detectable)."""
    o = pkg.default_options()
    assert o.struct_size == ctypes.sizeof(pkg.Options)


def test_noise_cache_limit_is_set_and_restored(pkg, built_lib):
    """ceemdan_noise_cache returns the previous limit; 0 disables (no device work involved)."""
    L = pkg.lib()
    prev = L.ceemdan_noise_cache(123456)
    try:
        assert L.ceemdan_noise_cache(789) == 123456
        assert L.ceemdan_noise_cache(0) == 789
    finally:
        L.ceemdan_noise_cache(prev)


def test_header_is_c99_and_links_alone(built_lib, tmp_path):
    """include/ceemdan_b200.h compiles as strict C99 and a C caller links against the library
    alone (the binding a C, cgo or FFI caller makes); host-rejected calls return their status
    without a device."""
    exe = tmp_path / "c_abi_caller"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi_caller.c"),
                    "-L", os.path.dirname(built_lib), "-lceemdan_b200",
                    "-Wl,-rpath," + os.path.dirname(built_lib), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["1", "1", "1", "1", "1", "0", "-1"]
