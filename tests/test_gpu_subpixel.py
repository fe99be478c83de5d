"""Conventional ptychography at sub-pixel scan positions: the CUDA library (C ABI) against the
FP64 oracle, the golden fixture composed from the reference's own functions, and central
finite differences.

Tolerance: relative L2 error 1e-5 for the loss and every gradient (FP64 references).
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


@pytest.fixture(scope="module", autouse=True)
def _lib():
    from ptychox_b200 import _abi

    _abi.load()
    assert torch.cuda.is_available()


def run_sweep(sample, probe, pos, meas, scale):
    from ptychox_b200.base import base_subpixel_sweep

    loss, gs, gp = base_subpixel_sweep(cuda(sample), cuda(probe), cuda(pos.astype(np.float64)), cuda(meas), scale)
    torch.cuda.synchronize()
    return float(loss.item()), gs.cpu().numpy(), gp.cpu().numpy()


def problem(n_obj, ph, pw, grid, step, origin, jitter, photons, seed, grid_x=None):
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    obj = synth.random_object(n_obj, n_obj, rng)
    probe = synth.gaussian_probe(ph, pw, rng)
    pos = synth.raster_positions_subpixel(grid, step, origin, jitter, rng, grid_x=grid_x)
    amp, _, _ = O.base_subpix_forward(obj, probe, pos, fp64=False)
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, photons, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    return guess, probe, pos, meas, scale


def test_sweep_golden():
    """The fixture composed from the reference's crop, shift_phase_ramp and ptychoX_base
    (rectangular 16 x 32 probe, real U[-2.5, 2.5] jitter)."""
    g = load_golden("sweep_base_subpix_fp64.npz")
    loss, gs, gp = run_sweep(g["sample"], g["probe"], g["positions"], g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL * abs(float(g["loss"]))
    assert rel_l2(gs, g["grad_sample"]) < TOL
    assert rel_l2(gp, g["grad_probe"]) < TOL


@pytest.mark.parametrize("ph,pw", [(32, 32), (64, 128), (128, 64), (256, 256)])
def test_sweep_vs_oracle_sizes(ph, pw):
    n = max(ph, pw) * 2 + 64
    guess, probe, pos, meas, scale = problem(n, ph, pw, 4, max(ph, pw) // 3, 20, 3.0, 1e4, seed=ph * 3 + pw)
    loss, gs, gp = run_sweep(guess, probe, pos, meas, scale)
    rl, rs, rp = O.base_subpix_sweep(guess, probe, pos, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL


def test_integer_positions_equal_the_integer_sweep():
    from ptychox_b200 import synth
    from ptychox_b200.base import base_sweep

    rng = np.random.default_rng(9)
    obj = synth.random_object(256, 256, rng)
    probe = synth.gaussian_probe(64, 64, rng)
    pos = synth.raster_positions(5, 40, 4, 2, rng)
    amp, _, _ = O.base_forward(obj, probe, pos)
    meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
    a = base_sweep(cuda(obj), cuda(probe), cuda(pos), cuda(meas), scale)
    loss, gs, gp = run_sweep(obj, probe, pos.astype(np.float64), meas, scale)
    assert abs(loss - float(a[0])) <= TOL * abs(float(a[0]))
    assert rel_l2(gs, a[1].cpu().numpy()) < TOL
    assert rel_l2(gp, a[2].cpu().numpy()) < TOL


def test_operator_matches_oracle_and_fused():
    """autograd.Function forward/backward vs the oracle, and F.mse_loss through it vs the fused loss."""
    from ptychox_b200 import ptychoX_base_subpixel, ptychoX_base_subpixel_loss

    guess, probe, pos, meas, scale = problem(256, 64, 32, 5, 30, 10, 2.0, 1e4, seed=23)
    # positions exactly representable in float32, so the float32 scan below is the same scan
    # (a float32 rounding of x ~ 100 moves it by up to 8e-6 px, a 1e-5 change of the gradient)
    pos = pos.astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(24)
    gout = rng.standard_normal((len(pos), 64, 32)).astype(np.float32)
    s = cuda(guess).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    amp = ptychoX_base_subpixel(s, p, torch.from_numpy(pos))  # host positions accepted
    (amp * cuda(gout)).sum().backward()
    ramp, far, shifted = O.base_subpix_forward(guess, probe, pos)
    rgs, rgp = O.base_subpix_backward(gout, shifted, probe.astype(np.complex128), far, pos, guess.shape)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(s.grad.cpu().numpy(), rgs) < TOL
    assert rel_l2(p.grad.cpu().numpy(), rgp) < TOL

    # F.mse_loss through the operator and the fused loss, each against the FP64 oracle sweep
    # (two FP32 paths differ from each other by up to the sum of their errors)
    rl, rs, rp = O.base_subpix_sweep(guess, probe, pos, meas, scale)
    _, fs, fp = O.base_subpix_sweep(guess, probe, pos, meas, scale, fp64=False)
    s2 = cuda(guess).requires_grad_(True)
    p2 = cuda(probe).requires_grad_(True)
    observed = torch.sqrt(cuda(meas).to(torch.float32) * np.float32(scale))
    torch.nn.functional.mse_loss(ptychoX_base_subpixel(s2, p2, cuda(pos)), observed).backward()
    s3 = cuda(guess).requires_grad_(True)
    p3 = cuda(probe).requires_grad_(True)
    loss3 = ptychoX_base_subpixel_loss(s3, p3, cuda(pos.astype(np.float32)), cuda(meas), scale)
    loss3.backward()
    assert abs(float(loss3.detach()) - rl) <= TOL * abs(rl)
    for g_s, g_p in ((s2.grad, p2.grad), (s3.grad, p3.grad)):
        assert rel_l2(g_s.cpu().numpy(), rs) < fp32_tol(rel_l2(fs, rs))
        assert rel_l2(g_p.cpu().numpy(), rp) < fp32_tol(rel_l2(fp, rp))


def test_windows_and_sizes_are_checked():
    import ptychox_b200
    from ptychox_b200 import ptychoX_base_subpixel

    s = torch.ones(64, 64, dtype=torch.complex64, device="cuda")
    p = torch.ones(16, 16, dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError, match="window leaves"):
        ptychoX_base_subpixel(s, p, torch.tensor([[48.6, 0.0]]))  # corner 49: 49 + 16 > 64
    ptychoX_base_subpixel(s, p, torch.tensor([[48.4, 0.0]]))  # corner 48 fits
    out = ptychoX_base_subpixel(s, p, torch.tensor([[-0.6, 0.0]], device="cuda"))  # device: deferred
    assert out.shape == (1, 16, 16)
    with pytest.raises(ValueError, match="window leaves the object"):
        ptychox_b200.check_errors()
    with pytest.raises(ValueError, match=r"2\^a 3\^b 5\^c"):
        ptychoX_base_subpixel(s, torch.ones(12, 16, dtype=torch.complex64, device="cuda"), torch.zeros(1, 2))


def _fd_subpixel(obj, probe, pos, meas, scale, obj_pix, probe_pix, delta=1e-5):
    """FP64 central differences of the oracle's loss at single object / probe pixels.

    Only the frames whose window covers the pixel change; their loss change is evaluated
    stably from FP64 far fields as (|F'| - |F|)(|F'| + |F| - 2Y)."""
    obj = obj.astype(np.complex128)
    probe = probe.astype(np.complex128)
    ph, pw = probe.shape
    amp0, far0, _ = O.base_subpix_forward(obj, probe, pos)
    y = O.measured_amplitude(meas, scale).astype(np.float64)
    numel = float(meas.size)
    corner, _ = O.subpixel_split(pos)

    def dloss(frames, o, pr):
        a1, f1, _ = O.base_subpix_forward(o, pr, pos[frames])
        a0 = amp0[frames]
        d = f1 - far0[frames]
        da = (2 * (np.conj(far0[frames]) * d).real + np.abs(d) ** 2) / (a1 + a0 + 1e-300)
        return float(np.sum(da * (a1 + a0 - 2 * y[frames]))) / numel

    fd_o = []
    for yy, xx in obj_pix:
        frames = [b for b, (x0, y0) in enumerate(corner.tolist()) if x0 <= xx < x0 + pw and y0 <= yy < y0 + ph]
        row = []
        for e in (1.0, 1j):
            op, om = obj.copy(), obj.copy()
            op[yy, xx] += delta * e
            om[yy, xx] -= delta * e
            row.append((dloss(frames, op, probe) - dloss(frames, om, probe)) / (2 * delta))
        fd_o.append(row)
    fd_p = []
    frames = list(range(len(pos)))
    for ly, lx in probe_pix:
        row = []
        for e in (1.0, 1j):
            pp, pm = probe.copy(), probe.copy()
            pp[ly, lx] += delta * e
            pm[ly, lx] -= delta * e
            row.append((dloss(frames, obj, pp) - dloss(frames, obj, pm)) / (2 * delta))
        fd_p.append(row)
    return np.array(fd_o), np.array(fd_p)


def test_config0_shape_vs_oracle_and_finite_differences():
    """Config 0 shape with real jitter (121 positions, 128^2 probe, 512^2 object, U[-2, 2]) against
    the FP64 oracle, and the fused loss's gradient against FP64 central differences of the
    oracle's loss at 48 object and 16 probe pixels."""
    from ptychox_b200 import ptychoX_base_subpixel_loss

    guess, probe, pos, meas, scale = problem(512, 128, 128, 11, 32, 8, 2.0, 1e4, seed=0)
    loss, gs, gp = run_sweep(guess, probe, pos, meas, scale)
    rl, rs, rp = O.base_subpix_sweep(guess, probe, pos, meas, scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL

    s = cuda(guess).requires_grad_(True)
    p = cuda(probe).requires_grad_(True)
    ptychoX_base_subpixel_loss(s, p, cuda(pos), cuda(meas), scale).backward()
    gs, gp = s.grad.cpu().numpy(), p.grad.cpu().numpy()
    rng = np.random.default_rng(5)
    corner, _ = O.subpixel_split(pos)
    obj_pix = [(int(y0 + rng.integers(8, 120)), int(x0 + rng.integers(8, 120)))
               for x0, y0 in corner[rng.choice(len(pos), 48, replace=False)].tolist()]
    probe_pix = [(int(a), int(b)) for a, b in rng.integers(40, 88, size=(16, 2))]
    fd_o, fd_p = _fd_subpixel(guess, probe, pos, meas, scale, obj_pix, probe_pix)
    g_o = np.array([[gs[y, x].real, gs[y, x].imag] for y, x in obj_pix])
    g_p = np.array([[gp[a, b].real, gp[a, b].imag] for a, b in probe_pix])
    assert rel_l2(g_o, fd_o) < TOL
    assert rel_l2(g_p, fd_p) < TOL


def test_config1_subpixel_subset_and_full():
    """Config 1 frames (2048^2 object, 512^2 probe, 30x30 raster step 48 with real U[-3, 3]
    jitter): a 48-position subset against the whole-batch FP64 oracle, then all 900 positions
    against the chunked FP64 oracle through the workspace the benchmark uses."""
    from ptychox_b200 import _abi, ptychoX_base_subpixel, synth
    from ptychox_b200._utils import workspace
    from ptychox_b200.base import base_subpixel_sweep

    rng = np.random.default_rng(1002)
    obj = synth.random_object(2048, 2048, rng)
    probe = synth.gaussian_probe(512, 512, rng)
    pos = synth.raster_positions_subpixel(30, 48, 64, 3.0, rng)
    with torch.no_grad():
        amp = ptychoX_base_subpixel(cuda(obj), cuda(probe), cuda(pos)).cpu().numpy()
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, 1e5, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)

    sub = rng.choice(len(pos), 48, replace=False)
    loss, gs, gp = run_sweep(guess, probe, pos[sub], meas[sub], scale)
    rl, rs, rp = O.base_subpix_sweep(guess, probe, pos[sub], meas[sub], scale)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(gs, rs) < TOL
    assert rel_l2(gp, rp) < TOL

    ws = workspace(_abi.query("ptx_base_subpix_workspace_bytes", 512, 512, len(pos)), torch.device("cuda"))
    loss, gs, gp = base_subpixel_sweep(cuda(guess), cuda(probe), cuda(pos), cuda(meas), scale, ws=ws)
    torch.cuda.synchronize()
    rl, rs, rp = O.base_subpix_sweep(guess, probe, pos, meas, scale, chunk=32, workers=O.default_workers())
    assert abs(float(loss.item()) - rl) <= TOL * abs(rl)
    assert rel_l2(gs.cpu().numpy(), rs) < TOL
    assert rel_l2(gp.cpu().numpy(), rp) < TOL
