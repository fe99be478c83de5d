"""Host-side check of the mixed-radix two-step register FFT for {2,3,5}-smooth lengths.

``ptx_mixfft.cuh`` writes each step of the transform as a per-thread ``__host__ __device__``
function, so the same steps the sweep kernels run can be executed on the CPU thread by
thread.  This test compiles ``mixfft_host.cu`` with nvcc as host code and checks every
smooth length from 6 to 1000 that is not a power of two, in both directions and both
exchange-buffer layouts, against an FP64 DFT at FP32 level.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "ptychox_b200" / "csrc"


def _smooth(n: int) -> bool:
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_mixed_radix_fft_matches_fp64_dft(tmp_path):
    exe = tmp_path / "mixfft_host"
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-x", "cu", "-Wno-deprecated-gpu-targets", "-I", str(CSRC),
                    str(HERE / "mixfft_host.cu"), "-o", str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [line.split() for line in out if line.strip()]
    want = [n for n in range(4, 1025) if _smooth(n)]
    assert [int(r[0]) for r in rows] == want
    for n, a, b, fwd, inv, ea, eb in rows:
        assert int(a) * int(b) == int(n) and int(a) <= int(b)
        # FP32 transforms: relative RMS error a few units of 2^-24 times log(n)
        assert float(fwd) < 3e-7 and float(inv) < 3e-7, (n, fwd, inv)
        assert float(ea) < 2e-7 and float(eb) < 2e-7, (n, ea, eb)
