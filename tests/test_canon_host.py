"""CPU checks of the engine's canonical arithmetic header (host-compiled)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_sx_filter_is_exact(tmp_path):
    exe = tmp_path / "sx_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    os.path.join(ROOT, "tests", "canon_sx_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0" in out.stdout


def test_reciprocal_division_is_exact(tmp_path):
    exe = tmp_path / "div_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    os.path.join(ROOT, "tests", "canon_div_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "mismatches 0" in out.stdout
