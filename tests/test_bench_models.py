"""The algorithmic byte models behind bench.py's roofline fractions, pinned to their per-sweep
values.

Conventional: per position 8 P^2 (patch gather) + 2 P^2 (uint16 counts) + 16 P^2 (object
gradient read-modify-write), per sweep + 16 P^2 (probe in, probe gradient out) + 8 N^2 (object
gradient zeroed).  Fourier: per LED 26 h^2, per sweep + 72 N^2 (the spectrum transform and
the inverse transform of its gradient, two global passes each, and the zeroing) + 16 h^2.
Coded / near-field: per position 240.125 N^2 (six 2-D transforms of two global passes each,
the mask and spectrum gradient updates, the stored forward field, the pooled counts), per
sweep + 64 N^2.
"""
import importlib.util
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_byte_models_per_sweep():
    w = load_bench().WORKLOADS
    p, n = 512.0, 2048.0
    assert w["conventional-900x512-2048"].bytes_per_sweep() == 26 * p * p * 900 + 16 * p * p + 8 * n * n
    assert round(w["conventional-900x512-2048"].bytes_per_sweep() / 1e6) == 6172  # 6.172 GB
    assert round(w["conventional-121x128-512"].bytes_per_sweep() / 1e5) == 539     # 53.9 MB
    assert round(w["fourier-225x256-1024"].bytes_per_sweep() / 1e6) == 460        # 0.460 GB
    assert round(w["coded-64x1024-ds4"].bytes_per_sweep() / 1e7) == 1618          # 16.18 GB
    assert w["nearfield-64x1024-ds4"].bytes_per_sweep() == w["coded-64x1024-ds4"].bytes_per_sweep()
