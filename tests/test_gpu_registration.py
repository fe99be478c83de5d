"""Sub-pixel registration on the GPU (``ptychox_b200.registration``, the upsampled-DFT
refinement in ``ptx_reg_upsampled_peak``) against the FP64 oracle
(``oracle/registration_oracle.py``, the restatement of ``dftregistration.m``).

Shifts: equal to the oracle's on the 1/usfac grid, or one grid step away where the two
neighbouring grid points differ in |CC| by less than FP32 can resolve (the FP32 and FP64
cross-correlations may then pick different neighbours).  Phase difference within 2e-4 and
squared error within 1e-5 (FP32 spectra and correlation sums against FP64).
"""

import numpy as np
import pytest
import torch

from oracle import registration_oracle as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from ptychox_b200 import _abi

    _abi.load()
    assert torch.cuda.is_available()


def smooth_image(h, w, rng, corr=0.2):
    f = np.fft.fft2(rng.standard_normal((h, w)))
    fy, fx = np.fft.fftfreq(h)[:, None], np.fft.fftfreq(w)[None, :]
    return np.real(np.fft.ifft2(f * np.exp(-(fx**2 + fy**2) / (2 * corr**2)))) + 3.0


def shifted(im, dy, dx):
    h, w = im.shape
    fy, fx = np.fft.fftfreq(h)[:, None], np.fft.fftfreq(w)[None, :]
    return np.real(np.fft.ifft2(np.fft.fft2(im) * np.exp(-2j * np.pi * (fy * dy + fx * dx))))


def check_rows(got, want, usfac):
    got, want = np.asarray(got), np.asarray(want)
    step = 1.0 / usfac if usfac > 0 else 0.0
    for g, w in zip(np.atleast_2d(got), np.atleast_2d(want)):
        # error = sqrt(1 - |CC|^2 / (E1 E2)): the FP32 sums fix 1 - |CC|^2 / (E1 E2) to about
        # 1e-6, which the square root amplifies near zero, so the bound is on error^2
        assert abs(g[0] ** 2 - w[0] ** 2) < 1e-5 and abs(g[1] - w[1]) < 2e-4
        for k in (2, 3):
            assert abs(g[k] - w[k]) <= step * 1.0001 + 1e-12


@pytest.mark.parametrize("usfac", [0, 1, 2, 3, 20, 100, 600])
@pytest.mark.parametrize("shape", [(48, 64), (45, 50)])
def test_dftregistration_matches_oracle(usfac, shape):
    from ptychox_b200.registration import dftregistration

    rng = np.random.default_rng(usfac * 7 + shape[1])
    h, w = shape
    im = smooth_image(h, w, rng)
    shifts = rng.uniform(-8, 8, size=(6, 2))
    stack = np.stack([shifted(im, dy, dx) + 0.005 * rng.standard_normal(im.shape) for dy, dx in shifts])
    b1 = np.fft.fft2(im)
    b2 = np.fft.fft2(stack, axes=(-2, -1))
    want = np.stack([R.dftregistration(b1, b, usfac) for b in b2])
    got = dftregistration(torch.from_numpy(b1).cuda(), torch.from_numpy(b2).cuda(), usfac).cpu().numpy()
    assert got.shape == (6, 4) and got.dtype == np.float64
    check_rows(got, want, usfac)
    one = dftregistration(torch.from_numpy(b1).cuda(), torch.from_numpy(b2[2]).cuda(), usfac).cpu().numpy()
    assert one.shape == (4,)
    check_rows(one, want[2], usfac)


@pytest.mark.parametrize("usfac", [0, 1, 100])
def test_registered_spectrum_matches_oracle(usfac):
    from ptychox_b200.registration import dftregistration, track_position

    rng = np.random.default_rng(40 + usfac)
    im = smooth_image(40, 56, rng)
    stack = np.stack([shifted(im, dy, dx) for dy, dx in rng.uniform(-5, 5, size=(3, 2))])
    b1, b2 = np.fft.fft2(im), np.fft.fft2(stack, axes=(-2, -1))
    out, greg = dftregistration(torch.from_numpy(b1).cuda(), torch.from_numpy(b2).cuda(), usfac,
                                return_registered=True)
    for k in range(3):
        # Greg from the GPU's own output, so only the FP32 spectrum and phase ramp differ
        want = R.registered(b2[k], out[k].cpu().numpy(), usfac)
        got = greg[k].cpu().numpy()
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-5
    if usfac == 100:
        big = np.stack([shifted(smooth_image(80, 80, rng, corr=0.3), 0, 0)] * 2)
        lx, ly, regi = track_position(torch.from_numpy(big).cuda(), usfac=usfac, return_registered=True)
        assert regi.shape == (2, 40, 40)


def test_track_and_refine_match_oracle():
    from ptychox_b200.registration import refine_position, track_position

    rng = np.random.default_rng(5)
    base = smooth_image(128, 144, rng, corr=0.3)
    shifts = rng.uniform(-6, 6, size=(8, 2))
    stack = np.stack([shifted(base, dy, dx) + 0.01 * rng.standard_normal(base.shape) for dy, dx in shifts])
    st = torch.from_numpy(stack).cuda()
    lx, ly = track_position(st)
    wx, wy = R.track_position(stack)
    assert np.abs(lx.cpu().numpy() - wx).max() <= 1.0001 / 600 and np.abs(ly.cpu().numpy() - wy).max() <= 1.0001 / 600
    rx, ry = refine_position(st, wx, wy)
    vx, vy = R.refine_position(stack, wx, wy)
    assert np.abs(rx.cpu().numpy() - vx).max() <= 1.0001 / 100 and np.abs(ry.cpu().numpy() - vy).max() <= 1.0001 / 100


def test_errors():
    from ptychox_b200 import _abi
    from ptychox_b200.registration import dftregistration, track_position

    z = torch.zeros(8, 8, dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        dftregistration(z, torch.zeros(8, 9, dtype=torch.complex64, device="cuda"))
    with pytest.raises(ValueError):
        dftregistration(z.cpu(), z.cpu())
    with pytest.raises(ValueError):
        dftregistration(z, z, -1)
    with pytest.raises(ValueError):
        track_position(torch.zeros(2, 30, 30, device="cuda"))
    assert _abi.query("ptx_reg_workspace_bytes", 4, 8, 8, 2) == 0
    assert _abi.query("ptx_reg_workspace_bytes", 1, 10, 12, 100) == 16 * 150 * (10 + 150)
