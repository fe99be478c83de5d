"""Fourier ptychography with sides that are not all powers of two (the mixed-radix FPM
kernels) against the FP64 oracle.

The reference takes any side (cuFFT and torch.fft); these cases cover even and odd smooth
sides, a power-of-two pupil in a smooth spectrum and the reverse, rectangular spectra and
pupils, windows that wrap around the spectrum edge or start at negative corners, the
fused sweep, the autograd operator (forward image and amplitude, backward) and a chunked
workspace.

Tolerance: relative L2 below 1e-5 for the loss, the amplitude and the object gradient.  The
pupil gradient carries the phase image/|image|, ill-conditioned at dark image pixels, so any
FP32 evaluation misses the FP64 value by an amount the problem sets (1e-5 to 1e-4 on these
scans, for the reference's own FP32 formulation too).  For power-of-two sides this build's
error tracks the reference FP32 error closely (ratio 1.0-1.2: both round like radix-2/4
passes), which is what ``fp32_tol`` (2x) assumes.  For other sides the two FP32 evaluations
factor the transforms differently and their rounding is uncorrelated: over 33 seeded scans
of this geometry on a B200 the ratio of this build's pupil-gradient error to the reference
FP32 error ranged 0.36-4.9 (median 1.1).  The bar for it is therefore 5x the reference FP32
error (at least 1e-5).
"""

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import ptycho_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module", autouse=True)
def _lib():
    import ptychox_b200  # noqa: F401
    from ptychox_b200 import _abi

    _abi.load()
    assert torch.cuda.is_available()


def problem(oh, ow, lh, lw, grid, seed, photons=5e3):
    """Random object; elliptical pupil (radius 0.3 of each side) with a random phase; a
    grid x grid LED layout stepping a fifth of the pupil around the centred window, plus
    three windows that wrap around the spectrum edge or start at negative corners."""
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    obj = synth.random_object(oh, ow, rng)
    yy, xx = np.meshgrid(np.arange(lh) - lh // 2, np.arange(lw) - lw // 2, indexing="ij")
    aperture = (((yy / (0.3 * lh)) ** 2 + (xx / (0.3 * lw)) ** 2) <= 1.0).astype(np.complex64)
    cx, cy, c = (ow - lw) // 2, (oh - lh) // 2, (grid - 1) // 2
    sx, sy = max(1, lw // 5), max(1, lh // 5)
    led = [[cx + (i - c) * sx, cy + (j - c) * sy] for j in range(grid) for i in range(grid)]
    led += [[-lw // 2, 3], [ow - lw // 3, oh - 5], [ow + 7, -9]]
    led = np.array(led, np.int64)
    amp, _, _ = O.fpm_forward(obj, aperture, led)
    meas, scale = synth.poisson_counts(amp**2, photons, rng, per_pixel=True, brightest=True)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    pup = (aperture * np.exp(0.2j * rng.standard_normal(aperture.shape))).astype(np.complex64)
    return guess, pup, led, meas, scale


def pupil_bar(err_reference_fp32):
    """Pupil-gradient bar for the mixed-radix path (see the module docstring)."""
    return max(TOL, 5.0 * err_reference_fp32)


def check_sweep(obj, pup, led, meas, scale, ws=None):
    from ptychox_b200.fpm import fpm_sweep

    loss, go, gp = fpm_sweep(cuda(obj), cuda(pup), cuda(led), cuda(meas), scale, ws=ws)
    torch.cuda.synchronize()
    rl, ro, rp = O.fpm_sweep(obj, pup, led, meas, scale)
    _, _, rp32 = O.fpm_sweep(obj, pup, led, meas, scale, fp64=False)
    assert abs(float(loss.item()) - rl) <= TOL * abs(rl)
    assert rel_l2(go.cpu().numpy(), ro) < TOL
    assert rel_l2(gp.cpu().numpy(), rp) < pupil_bar(rel_l2(rp32, rp))
    return float(loss.item()), go, gp


@pytest.mark.parametrize("oh,ow,lh,lw", [
    (200, 200, 40, 40),     # smooth spectrum and pupil
    (240, 240, 64, 64),     # power-of-two pupil in a smooth spectrum
    (256, 256, 60, 60),     # smooth pupil in a power-of-two spectrum
    (225, 225, 45, 45),     # odd sides (fftshift / ifftshift differ)
    (375, 375, 75, 75),
    (240, 200, 48, 40),     # rectangular
    (135, 320, 27, 64),     # odd rows, power-of-two columns
    (1000, 1000, 250, 250),
])
def test_sweep_generic_sides(oh, ow, lh, lw):
    check_sweep(*problem(oh, ow, lh, lw, 7 if max(oh, ow) <= 512 else 5, seed=oh * 7 + lw))


def test_config2_like_smooth_sizes():
    """Config 2's geometry at smooth non-power-of-two sides: a 960^2 spectrum, 240^2 pupil,
    13 x 13 LED grid (NA 0.1, pitch 4 mm, 90 mm), circular pupil."""
    from ptychox_b200 import synth

    rng = np.random.default_rng(5)
    n, h = 960, 240
    obj = synth.random_object(n, n, rng)
    pupil = synth.circular_pupil(h, 0.3)
    dx = synth.fpm_dx_for_pupil(n, h, 0.1, 0.532, 0.3)
    led = synth.fpm_led_windows(n, h, 13, 4.0, 90.0, 0.532, dx)
    amp, _, _ = O.fpm_forward(obj, pupil, led)
    meas, scale = synth.poisson_counts(amp**2, 5e3, rng, per_pixel=True, brightest=True)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    pup = (pupil * np.exp(0.2j * rng.standard_normal(pupil.shape))).astype(np.complex64)
    check_sweep(guess, pup, led, meas, scale)


@pytest.mark.parametrize("oh,ow,lh,lw", [(120, 120, 30, 30), (225, 200, 45, 50), (256, 240, 64, 48)])
def test_operator_forward_backward(oh, ow, lh, lw):
    """The autograd operator (forward: spectrum, rows, column forward mode; backward: column
    backward mode, adjoint rows, inverse spectrum transform) against the oracle, and the fused
    loss against the oracle's sweep."""
    from ptychox_b200 import ptychoX_fourier, ptychoX_fourier_loss

    obj, pup, led, meas, scale = problem(oh, ow, lh, lw, 5, seed=oh + lw)
    rng = np.random.default_rng(lh)
    gout = rng.standard_normal((len(led), lh, lw)).astype(np.float32)
    o = cuda(obj).requires_grad_(True)
    p = cuda(pup).requires_grad_(True)
    amp = ptychoX_fourier(o, p, torch.from_numpy(led))
    (amp * cuda(gout)).sum().backward()
    ramp, image, sub = O.fpm_forward(obj, pup, led)
    rgo, rgp = O.fpm_backward(gout, sub, pup.astype(np.complex128), image, led, obj.shape)
    # the backward's pupil gradient carries image/|image| too
    _, im32, sub32 = O.fpm_forward(obj, pup, led, fp64=False)
    _, gp32 = O.fpm_backward(gout, sub32, pup, im32, led, obj.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(o.grad.cpu().numpy(), rgo) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < pupil_bar(rel_l2(gp32, rgp))

    rl, ro, rp = O.fpm_sweep(obj, pup, led, meas, scale)
    o3 = cuda(obj).requires_grad_(True)
    p3 = cuda(pup).requires_grad_(True)
    loss = ptychoX_fourier_loss(o3, p3, cuda(led), cuda(meas), scale)
    loss.backward()
    assert abs(float(loss) - rl) <= TOL * abs(rl)
    assert rel_l2(o3.grad.cpu().numpy(), ro) < TOL
    _, _, rp32 = O.fpm_sweep(obj, pup, led, meas, scale, fp64=False)
    assert rel_l2(p3.grad.cpu().numpy(), rp) < pupil_bar(rel_l2(rp32, rp))


def test_chunked_workspace():
    """A workspace of two frames (many launch triples) matches the one-chunk sweep."""
    from ptychox_b200 import _abi
    from ptychox_b200.fpm import fpm_sweep

    obj, pup, led, meas, scale = problem(150, 150, 30, 30, 3, seed=21)
    loss, go, gp = check_sweep(obj, pup, led, meas, scale)
    lib = _abi.load()
    one = lib.ptx_fpm_workspace_bytes(150, 150, 30, 30, 1)
    frame = 2 * 16 * 30 * 8  # 30 columns -> 2 tiles of 16
    ws = torch.empty(one + frame, dtype=torch.uint8, device="cuda")
    l2, g2, p2 = fpm_sweep(cuda(obj), cuda(pup), cuda(led), cuda(meas), scale, ws=ws)
    assert abs(float(l2) - loss) <= 1e-12 * abs(loss)
    assert rel_l2(g2.cpu().numpy(), go.cpu().numpy()) < 1e-6
    assert rel_l2(p2.cpu().numpy(), gp.cpu().numpy()) < 1e-6


def test_unsupported_side_is_an_error():
    from ptychox_b200 import ptychoX_fourier

    o = torch.zeros(98, 98, dtype=torch.complex64, device="cuda")  # 98 = 2 * 7^2
    p = torch.zeros(14, 14, dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        ptychoX_fourier(o, p, torch.zeros(1, 2, dtype=torch.long))
