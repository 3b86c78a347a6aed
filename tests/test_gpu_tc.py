"""Tensor-core building blocks (gisspa_b200/csrc/tc.cuh) on a B200: a
tcgen05 GEMM with f32 inputs split into 16-bit (hi, lo) parts, against a
double-precision product (tests/native/test_tc_gemm.cu)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


def test_tcgen05_split_gemm(tmp_path):
    exe = str(tmp_path / "test_tc_gemm")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I" + os.path.join(ROOT, "gisspa_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "native", "test_tc_gemm.cu")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
