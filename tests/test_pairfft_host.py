"""Host-side check of the two-line packed-FP32x2 register FFT.

The transform in ``ptx_pairfft.cuh`` is written on ``__host__ __device__`` helpers, so the
same per-thread steps the column kernel runs can be executed on the CPU.  This test
compiles ``pairfft_host.cu`` with nvcc as host code, runs it for N = 4 .. 1024 in both
directions and bounds the error against an FP64 DFT at FP32 level.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "ptychox_b200" / "csrc"


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_pair_fft_matches_fp64_dft(tmp_path):
    exe = tmp_path / "pairfft_host"
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-x", "cu", "-I", str(CSRC), str(HERE / "pairfft_host.cu"),
                    "-o", str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [line.split() for line in out if line.strip()]
    assert [int(r[0]) for r in rows] == [4, 8, 16, 32, 64, 128, 256, 512, 1024]
    for n, fwd, inv in rows:
        # FP32 transform of length n: error grows like log2(n) * 2^-24
        assert float(fwd) < 3e-7 and float(inv) < 3e-7, (n, fwd, inv)
