"""The chunked FP64 oracle sweeps equal the whole-batch sweeps (CPU, small cases).

The full-size parity tests (config 1 at 900 positions, config 3 at 64 shifts) compare the
CUDA sweeps with these chunked sums, so the chunking itself is checked here first.
"""

import numpy as np

from conftest import rel_l2
from oracle import ptycho_oracle as O


def test_base_sweep_chunked_equals_whole():
    from ptychox_b200 import synth

    rng = np.random.default_rng(11)
    obj = synth.random_object(96, 96, rng)
    probe = synth.gaussian_probe(32, 32, rng)
    pos = synth.raster_positions(5, 12, 4, 2, rng)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
    whole = O.base_sweep(obj, probe, pos, meas, scale)
    chunk = O.base_sweep_chunked(obj, probe, pos, meas, scale, chunk=7)
    assert abs(chunk[0] - whole[0]) <= 1e-12 * abs(whole[0])
    assert rel_l2(chunk[1], whole[1]) < 1e-12
    assert rel_l2(chunk[2], whole[2]) < 1e-12


def test_coded_sweep_chunked_equals_whole():
    from ptychox_b200 import synth

    rng = np.random.default_rng(12)
    n = 32
    obj = synth.random_object(n, n, rng)
    mask = synth.binary_mask(n, 0.5, rng)
    t2 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 2e-3)
    t1 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 396.95e-6)
    shifts = synth.coded_shifts(10, 3.0, n, rng)
    for tr1 in (t1, None):
        _, _, _, amp = O.coded_forward(obj, mask, tr1, t2, shifts, 4)
        meas, scale = synth.poisson_counts(amp**2, 1e3, rng, per_pixel=True)
        whole = O.coded_sweep(obj, mask, tr1, t2, shifts, 4, meas, scale)
        chunk = O.coded_sweep_chunked(obj, mask, tr1, t2, shifts, 4, meas, scale, chunk=3)
        assert abs(chunk[0] - whole[0]) <= 1e-12 * abs(whole[0])
        assert rel_l2(chunk[1], whole[1]) < 1e-12
        assert rel_l2(chunk[2], whole[2]) < 1e-12
