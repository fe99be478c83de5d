"""Conventional sweep and operator on the mixed-radix register FFT kernels (the 2^a 3^b 5^c
line lengths 6..1000 that are not powers of two) against the FP64 oracle.

Covers square probes over the range of lengths (even and odd, tile-aligned and not),
rectangular probes whose rows and columns take different engines, the unfused forward and
backward operator passes (the column kernel's far-field and backward modes), chunked
workspaces and the window check.  Tolerance: relative L2 below 1e-5, the FP32 bar.
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


def problem(ph, pw, n_pos, seed, margin=24):
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    h, w = ph + 3 * margin + 8, pw + 3 * margin + 8
    obj = synth.random_object(h, w, rng)
    probe = synth.gaussian_probe(ph, pw, rng)
    pos = np.stack([rng.integers(0, w - pw + 1, n_pos), rng.integers(0, h - ph + 1, n_pos)], axis=1).astype(np.int64)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    return guess, probe, pos, meas, scale


def check_sweep(guess, probe, pos, meas, scale, ws=None):
    from ptychox_b200.base import base_sweep

    loss, gs, gp = base_sweep(cuda(guess), cuda(probe), cuda(pos), cuda(meas), scale, ws=ws)
    torch.cuda.synchronize()
    rl, rs, rp = O.base_sweep(guess, probe, pos, meas, scale)
    assert abs(float(loss.item()) - rl) <= TOL * abs(rl)
    assert rel_l2(gs.cpu().numpy(), rs) < TOL
    assert rel_l2(gp.cpu().numpy(), rp) < TOL
    return float(loss.item()), gs, gp


@pytest.mark.parametrize("p", [6, 12, 45, 75, 100, 120, 125, 150, 243, 375, 400, 480, 576, 600, 625, 640, 729, 810,
                               1000])
def test_square_sweep(p):
    from ptychox_b200 import _abi

    assert _abi.query("ptx_fft_engine", p) == 2
    n_pos = 4 if p <= 400 else 2
    check_sweep(*problem(p, p, n_pos, seed=p))


@pytest.mark.parametrize("ph,pw", [(100, 120), (120, 100), (45, 96), (96, 45), (640, 96), (96, 640), (125, 64),
                                   (64, 125), (384, 512), (512, 600), (30, 1000)])
def test_rectangular_sweep(ph, pw):
    """Rows and columns on different lengths and engines (mixed-radix with power-of-two)."""
    check_sweep(*problem(ph, pw, 3, seed=ph * 1009 + pw))


@pytest.mark.parametrize("ph,pw", [(96, 96), (75, 100), (160, 144), (640, 640)])
def test_operator_forward_backward(ph, pw):
    """The autograd operator: rows forward + column forward mode (far field and amplitude),
    then column backward mode + rows adjoint, against the oracle's forward and adjoint."""
    from ptychox_b200 import ptychoX_base

    guess, probe, pos, _, _ = problem(ph, pw, 3, seed=ph + 7 * pw)
    rng = np.random.default_rng(ph)
    gout = rng.standard_normal((len(pos), ph, pw)).astype(np.float32)
    s = cuda(guess).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    amp = ptychoX_base(s, p, cuda(pos))
    (amp * cuda(gout)).sum().backward()
    ramp, far, patches = O.base_forward(guess, probe, pos)
    rgs, rgp = O.base_backward(gout, patches, probe.astype(np.complex128), far, pos, guess.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(s.grad.cpu().numpy(), rgs) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < TOL


def test_chunked_workspace_and_many_frames():
    """A workspace of one frame (one launch triple per frame) equals the full workspace, and a
    scan of 60 frames (several adjoint frames per CTA) matches the oracle."""
    from ptychox_b200.base import base_sweep

    guess, probe, pos, meas, scale = problem(120, 120, 60, seed=11, margin=60)
    loss, gs, gp = check_sweep(guess, probe, pos, meas, scale)
    frame = 8 * 16 * 120 * 8  # 120 columns -> 8 tiles of 16
    ws = torch.empty(256 + 65536 * 4 + frame, dtype=torch.uint8, device="cuda")
    l1, g1, p1 = base_sweep(cuda(guess), cuda(probe), cuda(pos), cuda(meas), scale, ws=ws)
    assert abs(float(l1) - loss) <= 1e-12 * abs(loss)
    assert rel_l2(g1.cpu().numpy(), gs.cpu().numpy()) < 1e-6
    assert rel_l2(p1.cpu().numpy(), gp.cpu().numpy()) < 1e-6


def test_window_check_mixed_radix():
    """The mixed-radix forward row pass flags a window that leaves the object."""
    import ptychox_b200
    from ptychox_b200 import ptychoX_base

    s = torch.ones(200, 200, dtype=torch.complex64, device="cuda")
    p = torch.ones(96, 96, dtype=torch.complex64, device="cuda")
    ptychoX_base(s, p, torch.tensor([[0, 0], [150, 3]], device="cuda"))
    with pytest.raises(ValueError, match="window leaves the object"):
        ptychox_b200.check_errors()
    ptychoX_base(s, p, torch.tensor([[0, 0], [104, 104]], device="cuda"))
    ptychox_b200.check_errors()
