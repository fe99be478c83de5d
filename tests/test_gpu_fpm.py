"""Fourier ptychography: CUDA library (C ABI) vs the oracle and golden vectors.

Tolerance: relative L2 error below 1e-5 for loss and gradients (FP64 references).
"""

import numpy as np
import pytest
import torch

from conftest import fp32_tol, load_golden, rel_l2
from oracle import ptycho_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_sweep(obj, pupil, led, meas, scale):
    from ptychox_b200.fpm import fpm_sweep

    loss, go, gp = fpm_sweep(cuda(obj), cuda(pupil), cuda(led.astype(np.int64)), cuda(meas), scale)
    torch.cuda.synchronize()
    return float(loss.item()), go.cpu().numpy(), gp.cpu().numpy()


def test_test_ops_case():
    """python/test_ops.py:51-75 (16x16 object, 8x8 pupil)."""
    from ptychox_b200 import ptychoX_fourier

    g = load_golden("test_ops_fpm.npz")
    o = cuda(g["object"]).requires_grad_(True)
    p = cuda(g["pupil"]).requires_grad_(True)
    out = ptychoX_fourier(o, p, cuda(g["leds"]), use_cuda_kernels=True)
    (out * cuda(g["grad"])).sum().backward()
    assert rel_l2(out.detach().cpu().numpy(), g["out"]) < TOL
    assert rel_l2(o.grad.cpu().numpy(), g["grad_object"]) < TOL
    assert rel_l2(p.grad.cpu().numpy(), g["grad_pupil"]) < TOL


def pupil_tol(obj, pup, led, meas, scale, ref_gp):
    """Pupil-gradient tolerance: ``fp32_tol`` of the reference's own FP32 error here.

    grad_pupil carries the amplitude-loss phase image/|image|, ill-conditioned at dark
    image pixels in any FP32 evaluation.
    """
    _, _, gp32 = O.fpm_sweep(obj, pup, led, meas, scale, fp64=False)
    return fp32_tol(rel_l2(gp32, ref_gp))


def test_sweep_golden():
    g = load_golden("sweep_fpm_fp64.npz")
    loss, go, gp = run_sweep(g["object"], g["pupil"], g["leds"], g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL * abs(float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < TOL
    tol = pupil_tol(g["object"], g["pupil"], g["leds"], g["measured"], float(g["scale"]), g["grad_pupil"])
    assert rel_l2(gp, g["grad_pupil"]) < tol


def fpm_problem(n, h, grid, photons, seed, wrap=False):
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    obj = synth.random_object(n, n, rng)
    pupil = synth.circular_pupil(h, 0.3)
    dx = synth.fpm_dx_for_pupil(n, h, 0.1, 0.532, 0.3)
    led = synth.fpm_led_windows(n, h, grid, 4.0, 90.0, 0.532, dx)
    if wrap:  # windows crossing the spectrum edge and negative corners
        led = np.concatenate([led, np.array([[-h // 2, 3], [n - h // 3, n - 5], [n + 7, -9]], np.int64)])
    amp, _, _ = O.fpm_forward(obj, pupil, led)
    meas, scale = synth.poisson_counts(amp**2, photons, rng, per_pixel=True, brightest=True)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    pup = (pupil * np.exp(0.2j * rng.standard_normal(pupil.shape))).astype(np.complex64)
    return guess, pup, led, meas, scale


def test_config2_sweep_vs_oracle():
    """Config 2 shape: 1024x1024 spectrum, 15x15 LEDs, 256x256 pupil (NA 0.1, pitch 4 mm, 90 mm)."""
    obj, pup, led, meas, scale = fpm_problem(1024, 256, 15, 5e3, seed=2)
    assert led.shape == (225, 2)
    loss, go, gp = run_sweep(obj, pup, led, meas, scale)
    rl, ro, rp = O.fpm_sweep(obj, pup, led, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(go, ro) < TOL
    assert rel_l2(gp, rp) < pupil_tol(obj, pup, led, meas, scale, rp)


def test_wrapping_windows_and_operator():
    """Windows that wrap around the spectrum; autograd operator vs oracle and vs fused sweep."""
    from ptychox_b200 import ptychoX_fourier, ptychoX_fourier_loss

    obj, pup, led, meas, scale = fpm_problem(128, 32, 5, 200.0, seed=3, wrap=True)
    loss, go, gp = run_sweep(obj, pup, led, meas, scale)
    rl, ro, rp = O.fpm_sweep(obj, pup, led, meas, scale)
    ptol = pupil_tol(obj, pup, led, meas, scale, rp)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(go, ro) < TOL and rel_l2(gp, rp) < ptol

    rng = np.random.default_rng(9)
    gout = rng.standard_normal((len(led), 32, 32)).astype(np.float32)
    o = cuda(obj).requires_grad_(True)
    p = cuda(pup).requires_grad_(True)
    amp = ptychoX_fourier(o, p, torch.from_numpy(led))
    (amp * cuda(gout)).sum().backward()
    ramp, image, sub = O.fpm_forward(obj, pup, led)
    rgo, rgp = O.fpm_backward(gout, sub, pup.astype(np.complex128), image, led, obj.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(o.grad.cpu().numpy(), rgo) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < TOL

    o2 = cuda(obj).requires_grad_(True)
    p2 = cuda(pup).requires_grad_(True)
    ptychoX_fourier_loss(o2, p2, cuda(led), cuda(meas), scale).backward()
    assert abs(float(ptychoX_fourier_loss(cuda(obj), cuda(pup), cuda(led), cuda(meas), scale)) - rl) <= TOL * rl
    assert rel_l2(o2.grad.cpu().numpy(), ro) < TOL
    assert rel_l2(p2.grad.cpu().numpy(), rp) < ptol


def test_rectangular_and_unsupported():
    from ptychox_b200 import ptychoX_fourier

    rng = np.random.default_rng(4)
    obj = (rng.standard_normal((64, 128)) + 1j * rng.standard_normal((64, 128))).astype(np.complex64)
    pup = (rng.standard_normal((16, 32)) + 1j * rng.standard_normal((16, 32))).astype(np.complex64)
    led = np.array([[10, 5], [40, 20], [90, 40]], np.int64)
    amp = ptychoX_fourier(cuda(obj), cuda(pup), cuda(led))
    ramp, _, _ = O.fpm_forward(obj, pup, led)
    assert rel_l2(amp.cpu().numpy(), ramp) < TOL
    amp96 = ptychoX_fourier(cuda(obj[:, :96]), cuda(pup), cuda(led))  # 96 = 2^5 3: the mixed-radix path
    assert rel_l2(amp96.cpu().numpy(), O.fpm_forward(obj[:, :96], pup, led)[0]) < TOL
    with pytest.raises(ValueError):
        ptychoX_fourier(cuda(obj[:, :112]), cuda(pup), cuda(led))  # 112 = 2^4 7: no FFT length
