"""The in-register DFTs (radix 2-8 and 16, including the prime-factor radix 6
of the 1536-point tail pass), the radix-16 twiddle powers built from six
tabulated ones, and the compile-time pass plans of every specialised length, checked on the CPU: tests/host/fft_core_check.cu compiles
fft_core.cuh's host-and-device code for the host with nvcc and compares each
DFT with a direct FP64 sum."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc is not installed")
def test_dfts_and_plans_on_host(tmp_path):
    exe = tmp_path / "fft_core_check"
    subprocess.run([NVCC, "-std=c++17", "-O1", "-o", str(exe), os.path.join(HERE, "host", "fft_core_check.cu")],
                   check=True, capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout
    lines = out.stdout.strip().splitlines()
    assert len(lines) == 30 and all(l.endswith("ok") for l in lines), out.stdout
