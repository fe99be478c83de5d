"""Full-size parity: the benchmarked configurations in full against the FP64 oracle.

* Config 1 (900 positions, 512x512 probe, 2048x2048 object): the fused sweep through the
  same entry point and workspace size the benchmark uses, against the chunked FP64 oracle;
  and the autograd.Function gradient of the fused loss against FP64 central differences
  at 64 random pixels (48 of the object, 16 of the probe) over all 900 positions.
* Config 3 (64 shifts of a 1024x1024 field, ds 4), coded and near-field, in full.

Tolerance: relative L2 error 1e-5 for the loss and every gradient; where the reference's
own FP32 formulation (the oracle in complex64) misses 1e-5 on the same inputs, twice that
error (``conftest.fp32_tol``).  The oracle's whole-batch arrays would take several GB here,
so it accumulates over chunks of positions (checked against the whole-batch oracle in
``test_oracle_chunked.py``).
"""

import numpy as np
import pytest
import torch

from conftest import fp32_tol, rel_l2
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


@pytest.fixture(scope="module")
def config1():
    """Config 1 problem: counts from the forward model of the truth (Poisson, 1e5 photons per
    pattern, uint16), the sweep evaluated at the truth perturbed by 10% complex noise."""
    from ptychox_b200 import ptychoX_base, synth

    rng = np.random.default_rng(1001)
    obj = synth.random_object(2048, 2048, rng)
    probe = synth.gaussian_probe(512, 512, rng)
    pos = synth.raster_positions(30, 48, 64, 3, rng)
    assert len(pos) == 900
    with torch.no_grad():
        amp = ptychoX_base(cuda(obj), cuda(probe), cuda(pos)).cpu().numpy()
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, 1e5, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    return guess, probe, pos, meas, scale


def test_config1_full_sweep_vs_oracle(config1):
    """All 900 positions in one sweep with the benchmark's workspace (one chunk of 900 frames)."""
    from ptychox_b200 import _abi
    from ptychox_b200._utils import workspace
    from ptychox_b200.base import base_sweep

    guess, probe, pos, meas, scale = config1
    ws = workspace(_abi.query("ptx_base_workspace_bytes", 512, 512, len(pos)), torch.device("cuda"))
    loss, gs, gp = base_sweep(cuda(guess), cuda(probe), cuda(pos), cuda(meas), scale, ws=ws)
    torch.cuda.synchronize()
    rl, rs, rp = O.base_sweep_chunked(guess, probe, pos, meas, scale, chunk=32, workers=O.default_workers())
    assert abs(float(loss.item()) - rl) <= TOL * abs(rl)
    assert rel_l2(gs.cpu().numpy(), rs) < TOL
    assert rel_l2(gp.cpu().numpy(), rp) < TOL


def _fd_pixels(obj, probe, pos, meas, scale, obj_pix, probe_pix, delta=1e-5, chunk=30, device="cuda"):
    """FP64 central differences of the amplitude-MSE loss at single object and probe pixels,
    over all positions.

    A pixel perturbation changes each affected exit wave at one point, so that frame's far
    field changes by ``delta * value * (outer product of two DFT rows)``; the loss change is
    evaluated exactly from FP64 far fields, stably as (|F+D| - |F|)(|F+D| + |F| - 2Y) with
    |F+D| - |F| = (2 Re(conj(F) D) + |D|^2) / (|F+D| + |F|).  The far fields are formed in
    complex128 by torch (cuFFT Z2Z), one chunk of positions at a time, so the 900 x 512^2
    frames need not be held at once.  Returns (dL/dRe, dL/dIm) per pixel.
    """
    dev = torch.device(device)
    p = probe.shape[0]
    objt = torch.from_numpy(obj.astype(np.complex128)).to(dev)
    probet = torch.from_numpy(probe.astype(np.complex128)).to(dev)
    y_all = torch.from_numpy(O.measured_amplitude(meas, scale).astype(np.float64)).to(dev)
    numel = float(meas.size)
    k = torch.arange(p, dtype=torch.float64, device=dev) - p // 2

    def rows(l):
        return torch.exp(-2j * np.pi * k[None, :] * l[:, None].to(torch.float64) / p)

    def dloss(F, a, y, dF):
        anew = (F + dF).abs()
        diff = (2 * (F.conj() * dF).real + dF.abs() ** 2) / (anew + a + 1e-300)
        return float((diff * (anew + a - 2 * y)).sum())

    fd_o = np.zeros((len(obj_pix), 2))
    fd_p = np.zeros((len(probe_pix), 2))
    for b0 in range(0, len(pos), chunk):
        cp = pos[b0:b0 + chunk]
        patches = torch.stack([objt[y0:y0 + p, x0:x0 + p] for x0, y0 in cp.tolist()])
        F = torch.fft.fftshift(torch.fft.fft2(patches * probet[None]), dim=(-2, -1))
        a = F.abs()
        y = y_all[b0:b0 + chunk]
        x0 = torch.from_numpy(np.ascontiguousarray(cp[:, 0])).to(dev)
        y0 = torch.from_numpy(np.ascontiguousarray(cp[:, 1])).to(dev)
        for i, (yy, xx) in enumerate(obj_pix):
            sel = ((x0 <= xx) & (xx < x0 + p) & (y0 <= yy) & (yy < y0 + p)).nonzero().flatten()
            if sel.numel() == 0:
                continue
            ly, lx = yy - y0[sel], xx - x0[sel]
            v = probet[ly, lx]
            E = rows(ly)[:, :, None] * rows(lx)[:, None, :] * v[:, None, None]
            for j, e in enumerate((1.0, 1j)):
                plus = dloss(F[sel], a[sel], y[sel], delta * e * E)
                minus = dloss(F[sel], a[sel], y[sel], -delta * e * E)
                fd_o[i, j] += (plus - minus) / (2 * delta * numel)
        for i, (ly, lx) in enumerate(probe_pix):
            v = objt[y0 + ly, x0 + lx]
            lyv = torch.full_like(y0, ly)
            lxv = torch.full_like(x0, lx)
            E = rows(lyv)[:, :, None] * rows(lxv)[:, None, :] * v[:, None, None]
            for j, e in enumerate((1.0, 1j)):
                plus = dloss(F, a, y, delta * e * E)
                minus = dloss(F, a, y, -delta * e * E)
                fd_p[i, j] += (plus - minus) / (2 * delta * numel)
    return fd_o, fd_p


def test_config1_full_finite_differences(config1):
    """Config 1 at all 900 positions: the autograd.Function gradient of the fused loss vs FP64
    central differences at 64 random pixels (48 object pixels inside the scanned area, 16 probe
    pixels inside the probe's support)."""
    from ptychox_b200 import ptychoX_base_loss

    guess, probe, pos, meas, scale = config1
    s = cuda(guess).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    ptychoX_base_loss(s, p, cuda(pos), cuda(meas), scale).backward()
    gs, gp = s.grad.cpu().numpy(), p.grad.cpu().numpy()
    rng = np.random.default_rng(77)
    obj_pix = [(int(y0 + rng.integers(0, 512)), int(x0 + rng.integers(0, 512)))
               for x0, y0 in pos[rng.choice(len(pos), 48, replace=False)].tolist()]
    probe_pix = [(int(a), int(b)) for a, b in rng.integers(150, 362, size=(16, 2))]
    fd_o, fd_p = _fd_pixels(guess, probe, pos, meas, scale, obj_pix, probe_pix)
    g_o = np.array([[gs[y, x].real, gs[y, x].imag] for y, x in obj_pix])
    g_p = np.array([[gp[a, b].real, gp[a, b].imag] for a, b in probe_pix])
    assert rel_l2(g_o, fd_o) < TOL
    assert rel_l2(g_p, fd_p) < TOL


@pytest.mark.parametrize("nearfield", [False, True])
def test_config3_full_vs_oracle(nearfield):
    """Config 3 in full: 1024x1024 field at 1.85 um, lambda 0.5 um, z 2 mm (coded: T1 at
    396.95 um), 50% binary mask, 64 shifts U[-20, 20] px, ds 4, Poisson counts."""
    from ptychox_b200 import ptychoX_coded, ptychoX_nearfield, synth
    from ptychox_b200.coded import coded_sweep

    rng = np.random.default_rng(3003 + int(nearfield))
    n = 1024
    obj = synth.random_object(n, n, rng)
    mask = synth.binary_mask(n, 0.5, rng)
    t2 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 2e-3)
    t1 = None if nearfield else synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 396.95e-6)
    shifts = synth.coded_shifts(64, 20.0, n, rng).astype(np.float32)
    with torch.no_grad():
        if nearfield:
            amp = ptychoX_nearfield(cuda(obj), cuda(mask), cuda(t2), cuda(shifts), 4)
        else:
            amp = ptychoX_coded(cuda(obj), cuda(mask), cuda(t1), cuda(t2), cuda(shifts), 4)
    meas, scale = synth.poisson_counts(amp.cpu().numpy().astype(np.float64) ** 2, 2e3, rng, per_pixel=True)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    loss, go, gm = coded_sweep(cuda(guess), cuda(mask), None if t1 is None else cuda(t1), cuda(t2), cuda(shifts), 4,
                               cuda(meas), scale)
    torch.cuda.synchronize()
    go, gm = go.cpu().numpy(), gm.cpu().numpy()
    workers = O.default_workers()
    rl, ro, rm = O.coded_sweep_chunked(guess, mask, t1, t2, shifts, 4, meas, scale, chunk=8, workers=workers)
    assert abs(float(loss.item()) - rl) <= TOL * abs(rl)
    err_o, err_m = rel_l2(go, ro), rel_l2(gm, rm)
    if err_o >= TOL or err_m >= TOL:
        # FP32 itself limits accuracy here: the bar is twice the reference FP32 formulation's error
        _, o32, m32 = O.coded_sweep_chunked(guess, mask, t1, t2, shifts, 4, meas, scale, chunk=8, fp64=False,
                                            workers=workers)
        assert err_o < fp32_tol(rel_l2(o32, ro))
        assert err_m < fp32_tol(rel_l2(m32, rm))
