"""The registration oracle (``oracle/registration_oracle.py``) against the defining
properties of ``dftregistration.m`` (no MATLAB runs here to pin it to):

* an image shifted by a known sub-pixel amount (a Fourier phase ramp, exact for a periodic
  image) registers to minus that shift, to within half a grid step of 1/usfac;
* the usfac = 1 and usfac = 2 branches pick the maximum of the circular cross-correlation
  evaluated by a direct DFT sum on the integer / half-pixel grid;
* error 0 and the phase of a constant factor for a scaled copy; usfac = 0 gives the same
  error and phase without a shift;
* ``track_position`` / ``refine_position`` recover the shifts of a synthetic stack.
"""

import numpy as np
import pytest

from oracle import registration_oracle as R


def smooth_image(h, w, rng, corr=0.08):
    f = np.fft.fft2(rng.standard_normal((h, w)))
    fy, fx = np.fft.fftfreq(h)[:, None], np.fft.fftfreq(w)[None, :]
    return np.real(np.fft.ifft2(f * np.exp(-(fx**2 + fy**2) / (2 * corr**2)))) + 3.0


def shifted(im, dy, dx):
    h, w = im.shape
    fy, fx = np.fft.fftfreq(h)[:, None], np.fft.fftfreq(w)[None, :]
    return np.real(np.fft.ifft2(np.fft.fft2(im) * np.exp(-2j * np.pi * (fy * dy + fx * dx))))


@pytest.mark.parametrize("usfac", [3, 20, 100, 101, 600])
def test_recovers_known_subpixel_shifts(usfac):
    rng = np.random.default_rng(usfac)
    im = smooth_image(48, 64, rng)
    for _ in range(4):
        dy, dx = rng.uniform(-9, 9, 2)
        out = R.dftregistration(np.fft.fft2(im), np.fft.fft2(shifted(im, dy, dx)), usfac)
        assert abs(out[2] + dy) <= 0.5 / usfac + 2e-3 and abs(out[3] + dx) <= 0.5 / usfac + 2e-3
        assert out[0] < 1e-2


def _direct_cc(b1, b2, sy, sx):
    h, w = b1.shape
    ky = np.fft.fftfreq(h)[:, None] * h
    kx = np.fft.fftfreq(w)[None, :] * w
    return np.sum(b1 * np.conj(b2) * np.exp(2j * np.pi * (ky * sy / h + kx * sx / w)))


@pytest.mark.parametrize("usfac", [1, 2])
def test_integer_and_half_pixel_branches_match_direct_correlation(usfac):
    rng = np.random.default_rng(7 + usfac)
    im = smooth_image(16, 20, rng, corr=0.2)
    im2 = shifted(im, 2.3, -3.6) + 0.01 * rng.standard_normal(im.shape)
    b1, b2 = np.fft.fft2(im), np.fft.fft2(im2)
    out = R.dftregistration(b1, b2, usfac)
    step = 1.0 / usfac
    grid_y = np.arange(-8, 8, step)
    grid_x = np.arange(-10, 10, step)
    vals = np.array([[abs(_direct_cc(b1, b2, sy, sx)) for sy in grid_y] for sx in grid_x]).T
    iy, ix = np.unravel_index(np.argmax(vals), vals.shape)
    assert out[2] == pytest.approx(grid_y[iy]) and out[3] == pytest.approx(grid_x[ix])


def test_error_and_phase_of_a_scaled_copy():
    rng = np.random.default_rng(3)
    b1 = np.fft.fft2(smooth_image(32, 32, rng))
    b2 = b1 * 0.7 * np.exp(-1j * 0.9)
    for usfac in (0, 1, 2, 50):
        out = R.dftregistration(b1, b2, usfac)
        assert out[0] == pytest.approx(0.0, abs=1e-6)
        assert out[1] == pytest.approx(0.9, abs=1e-9)
        assert out[2] == 0.0 and out[3] == 0.0


def test_track_and_refine_recover_stack_shifts():
    # textured images: the 20-pixel border crop makes the windows differ at their edges,
    # which biases a broad correlation peak towards zero; a fine texture keeps it sharp
    rng = np.random.default_rng(11)
    base = smooth_image(160, 160, rng, corr=0.3)
    shifts = rng.uniform(-6, 6, size=(6, 2))
    shifts[0] = 0.0
    stack = np.stack([shifted(base, dy, dx) for dy, dx in shifts])
    lx, ly = R.track_position(stack, usfac=100)
    assert np.allclose(-lx, shifts[:, 1], atol=0.05) and np.allclose(-ly, shifts[:, 0], atol=0.05)
    rx, ry = R.refine_position(stack, lx, ly, usfac=100)
    # the refined reference is the stack average shifted back, so shifts are relative to it
    d = (-rx - shifts[:, 1]) - np.mean(-rx - shifts[:, 1])
    e = (-ry - shifts[:, 0]) - np.mean(-ry - shifts[:, 0])
    assert np.abs(d).max() < 0.1 and np.abs(e).max() < 0.1
