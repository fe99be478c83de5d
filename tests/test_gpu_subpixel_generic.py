"""Conventional ptychography at sub-pixel scan positions with probe sides that are
{2,3,5}-smooth but not powers of two (the mixed-radix sub-pixel kernels; a rectangular probe
may mix them with power-of-two sides) against the FP64 oracle.

Cases: even and odd sides, sides that 16 does not divide, rectangular probes mixing the two
engines, the fused sweep, the autograd operator (forward and backward), integer positions
against the integer sweep, and a chunked workspace.  Tolerance: relative L2 below 1e-5 (FP64
references).
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
    from ptychox_b200 import _abi

    _abi.load()
    assert torch.cuda.is_available()


def problem(ph, pw, n_pos, seed):
    """Random object and probe, `n_pos` float positions anywhere the window fits."""
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    h, w = ph + 3 * 24 + 8, pw + 3 * 24 + 8
    obj = synth.random_object(h, w, rng)
    probe = synth.gaussian_probe(ph, pw, rng)
    pos = np.stack([rng.uniform(0.0, w - pw - 0.51, n_pos), rng.uniform(0.0, h - ph - 0.51, n_pos)], axis=1)
    amp, _, _ = O.base_subpix_forward(obj, probe, pos, fp64=False)
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, 1e4, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    return guess, probe, pos, meas, scale


def run_sweep(sample, probe, pos, meas, scale, ws=None):
    from ptychox_b200.base import base_subpixel_sweep

    loss, gs, gp = base_subpixel_sweep(cuda(sample), cuda(probe), cuda(pos.astype(np.float64)), cuda(meas), scale,
                                       ws=ws)
    torch.cuda.synchronize()
    return float(loss.item()), gs.cpu().numpy(), gp.cpu().numpy()


@pytest.mark.parametrize("ph,pw", [(96, 96), (120, 100), (75, 75), (45, 64), (64, 90), (240, 240), (512, 600),
                                   (640, 640)])
def test_sweep_vs_oracle(ph, pw):
    guess, probe, pos, meas, scale = problem(ph, pw, 5 if max(ph, pw) <= 256 else 3, seed=ph * 11 + pw)
    loss, gs, gp = run_sweep(guess, probe, pos, meas, scale)
    rl, rs, rp = O.base_subpix_sweep(guess, probe, pos, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL


def test_operator_matches_oracle():
    """autograd.Function forward (column shift, row pass, column forward mode) and backward
    (shift-only rows, column backward mode, adjoint rows, column scatter) against the oracle."""
    from ptychox_b200 import ptychoX_base_subpixel

    guess, probe, pos, _, _ = problem(120, 100, 4, seed=7)
    pos = pos.astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(8)
    gout = rng.standard_normal((len(pos), 120, 100)).astype(np.float32)
    s = cuda(guess).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    amp = ptychoX_base_subpixel(s, p, torch.from_numpy(pos))
    (amp * cuda(gout)).sum().backward()
    ramp, far, shifted = O.base_subpix_forward(guess, probe, pos)
    rgs, rgp = O.base_subpix_backward(gout, shifted, probe.astype(np.complex128), far, pos, guess.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(s.grad.cpu().numpy(), rgs) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < TOL


def test_integer_positions_equal_the_integer_sweep():
    from ptychox_b200.base import base_sweep

    guess, probe, pos, meas, scale = problem(96, 120, 6, seed=9)
    pos = np.floor(pos).astype(np.int64)
    amp, _, _ = O.base_forward(guess, probe, pos)
    a = base_sweep(cuda(guess), cuda(probe), cuda(pos), cuda(meas), scale)
    loss, gs, gp = run_sweep(guess, probe, pos.astype(np.float64), meas, scale)
    assert abs(loss - float(a[0])) <= TOL * abs(float(a[0]))
    assert rel_l2(gs, a[1].cpu().numpy()) < TOL
    assert rel_l2(gp, a[2].cpu().numpy()) < TOL


def test_chunked_workspace():
    """A workspace of one frame pair (many launch sequences) matches the one-chunk sweep."""
    from ptychox_b200 import _abi

    guess, probe, pos, meas, scale = problem(75, 100, 5, seed=31)
    l1, g1, p1 = run_sweep(guess, probe, pos, meas, scale)
    hdr_and_ramps = _abi.query("ptx_base_subpix_workspace_bytes", 75, 100, 5) - 5 * 2 * (7 * 16 * 75 * 8)
    ws = torch.empty(hdr_and_ramps + 2 * (7 * 16 * 75 * 8), dtype=torch.uint8, device="cuda")
    l2, g2, p2 = run_sweep(guess, probe, pos, meas, scale, ws=ws)
    assert abs(l2 - l1) <= 1e-12 * abs(l1)
    assert rel_l2(g2, g1) < 1e-6 and rel_l2(p2, p1) < 1e-6
