"""Builds and runs the CPU harness of the Stockham passes (csrc/fft_core.cuh)."""
import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_stockham_passes_match_direct_dft(tmp_path):
    cxx = shutil.which("g++") or "/usr/bin/g++"
    exe = tmp_path / "fft_core_test"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "pandora-2.0_b200", "csrc"),
                    os.path.join(ROOT, "tests", "native", "fft_core_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
