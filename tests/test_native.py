"""Host-compiled checks of device code that also runs on the CPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_register_fft_against_double_dft(tmp_path):
    exe = str(tmp_path / "test_regfft")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "--expt-relaxed-constexpr",
                    "-Wno-deprecated-gpu-targets", "-I" + os.path.join(ROOT, "gisspa_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "native", "test_regfft.cu")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_prime_factor_maps_of_window_720(tmp_path):
    exe = str(tmp_path / "test_pfa")
    # device code of the included kernels is compiled for sm_100a (FP64 atomics);
    # only the host part runs
    subprocess.run(["nvcc", "-std=c++17", "-O2", "--expt-relaxed-constexpr",
                    "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "gisspa_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "native", "test_pfa.cu")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
