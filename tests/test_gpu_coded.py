"""Coded and near-field ptychography: CUDA library (C ABI) vs the oracle and golden vectors.

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


def run_sweep(obj, mask, t1, t2, shifts, ds, meas, scale, loss="mse"):
    from ptychox_b200.coded import coded_sweep

    loss, go, gm = coded_sweep(cuda(obj), cuda(mask), None if t1 is None else cuda(t1), cuda(t2),
                               cuda(shifts.astype(np.float32)), ds, cuda(meas), scale, loss=loss)
    torch.cuda.synchronize()
    return float(loss.item()), go.cpu().numpy(), gm.cpu().numpy()


def test_test_ops_case():
    """python/test_ops.py:77-104 (16x16, random transfer functions, ds=2)."""
    from ptychox_b200 import ptychoX_coded

    g = load_golden("test_ops_coded.npz")
    o = cuda(g["object"]).requires_grad_(True)
    m = cuda(g["mask"]).requires_grad_(True)
    out = ptychoX_coded(o, m, cuda(g["transfer_1"]), cuda(g["transfer_2"]), cuda(g["shifts"]), 2,
                        use_cuda_kernels=True)
    (out * cuda(g["grad"])).sum().backward()
    assert rel_l2(out.detach().cpu().numpy(), g["out"]) < TOL
    assert rel_l2(o.grad.cpu().numpy(), g["grad_object"]) < TOL
    assert rel_l2(m.grad.cpu().numpy(), g["grad_mask"]) < TOL


@pytest.mark.parametrize("name", ["sweep_coded_fp64.npz", "sweep_nearfield_fp64.npz"])
def test_sweep_golden(name):
    g = load_golden(name)
    t1 = None if bool(g["nearfield"]) else g["transfer_1"]
    loss, go, gm = run_sweep(g["object"], g["mask"], t1, g["transfer_2"], g["shifts"], int(g["downsample"]),
                             g["measured"], float(g["scale"]))
    assert abs(loss - float(g["loss"])) <= TOL * abs(float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < TOL
    assert rel_l2(gm, g["grad_mask"]) < TOL


def coded_problem(n, count, max_px, ds, photons, seed, nearfield):
    from ptychox_b200 import synth

    rng = np.random.default_rng(seed)
    obj = synth.random_object(n, n, rng)
    mask = synth.binary_mask(n, 0.5, rng)
    dx = 1.85e-6
    t2 = synth.angular_spectrum_transfer(n, dx, 0.5e-6, 2e-3)
    t1 = None if nearfield else synth.angular_spectrum_transfer(n, dx, 0.5e-6, 396.95e-6)
    shifts = synth.coded_shifts(count, max_px, n, rng)
    _, _, _, amp = O.coded_forward(obj, mask, t1, t2, shifts, ds, fp64=False)
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, photons, rng, per_pixel=True)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    return guess, mask, t1, t2, shifts, meas, scale


@pytest.mark.parametrize("nearfield", [False, True])
def test_config3_field_vs_oracle(nearfield):
    """Config 3 field: 1024x1024 at 1.85 um, lambda 0.5 um, z 2 mm, 50% binary mask, U[-20,20] px
    shifts, ds 4 -- on a 16-shift subset (the FP64 oracle holds whole-batch arrays)."""
    obj, mask, t1, t2, shifts, meas, scale = coded_problem(1024, 16, 20.0, 4, 2e3, seed=5, nearfield=nearfield)
    loss, go, gm = run_sweep(obj, mask, t1, t2, shifts, 4, meas, scale)
    rl, ro, rm = O.coded_sweep(obj, mask, t1, t2, shifts, 4, meas, scale)
    _, o32, m32 = O.coded_sweep(obj, mask, t1, t2, shifts, 4, meas, scale, fp64=False)
    assert abs(loss - rl) <= TOL * abs(rl)
    assert rel_l2(go, ro) < fp32_tol(rel_l2(o32, ro))
    assert rel_l2(gm, rm) < fp32_tol(rel_l2(m32, rm))


def test_operator_matches_oracle_and_fused():
    from ptychox_b200 import ptychoX_coded, ptychoX_coded_loss, ptychoX_nearfield

    obj, mask, t1, t2, shifts, meas, scale = coded_problem(128, 6, 5.0, 2, 500.0, seed=6, nearfield=False)
    rng = np.random.default_rng(8)
    gout = rng.standard_normal((6, 64, 64)).astype(np.float32)
    o = cuda(obj).requires_grad_(True)
    m = cuda(mask).requires_grad_(True)
    amp = ptychoX_coded(o, m, cuda(t1), cuda(t2), torch.from_numpy(shifts), 2)
    (amp * cuda(gout)).sum().backward()
    _, xf, sensor, ramp = O.coded_forward(obj, mask, t1, t2, shifts, 2)
    rgo, rgm = O.coded_backward(gout, xf, sensor, ramp, mask, t1, t2, shifts, 2)
    assert rel_l2(amp.detach().cpu().numpy(), ramp) < TOL
    assert rel_l2(o.grad.cpu().numpy(), rgo) < TOL
    assert rel_l2(m.grad.cpu().numpy(), rgm) < TOL

    rl, ro, rm = O.coded_sweep(obj, mask, t1, t2, shifts, 2, meas, scale)
    o2 = cuda(obj).requires_grad_(True)
    m2 = cuda(mask).requires_grad_(True)
    loss = ptychoX_coded_loss(o2, m2, cuda(t1), cuda(t2), cuda(shifts), 2, cuda(meas), scale)
    loss.backward()
    assert abs(float(loss.detach()) - rl) <= TOL * rl
    assert rel_l2(o2.grad.cpu().numpy(), ro) < TOL
    assert rel_l2(m2.grad.cpu().numpy(), rm) < TOL

    # near-field operator == coded operator with transfer_1 = 1
    ones = torch.ones(128, 128, dtype=torch.complex64, device="cuda")
    a1 = ptychoX_nearfield(cuda(obj), cuda(mask), cuda(t2), cuda(shifts), 2)
    a2 = ptychoX_coded(cuda(obj), cuda(mask), ones, cuda(t2), cuda(shifts), 2)
    assert rel_l2(a1.cpu().numpy(), a2.cpu().numpy()) < 1e-6


def test_input_errors():
    from ptychox_b200 import ptychoX_coded

    z = torch.zeros(64, 64, dtype=torch.complex64, device="cuda")
    sh = torch.zeros(2, 2, device="cuda")
    with pytest.raises(ValueError, match="same shape"):
        ptychoX_coded(z, z[:32], z, z, sh, 2)
    with pytest.raises(ValueError, match="divisible"):
        ptychoX_coded(z, z, z, z, sh, 3)
    with pytest.raises(ValueError, match=r"shape \[batch, 2\]"):
        ptychoX_coded(z, z, z, z, sh[:, :1], 2)
    w = torch.zeros(112, 112, dtype=torch.complex64, device="cuda")
    with pytest.raises(ValueError):
        ptychoX_coded(w, w, w, w, sh, 2)  # 112 = 2^4 7: no FFT length


@pytest.mark.parametrize("name,loss", [("sweep_coded_fd_iso_fp64.npz", "fd-isotropic"),
                                       ("sweep_coded_fd_aniso_fp64.npz", "fd-anisotropic")])
def test_fd_loss_golden(name, loss):
    """fd_loss (train_coded.py:101-107) through ptx_coded_sweep_fd against the reference's
    own loss and gradients.  Bar: 1e-5, or twice the error of the reference's FP32
    formulation where FP32 itself limits the result (the loss differences amplify the FP32
    error of the pooled amplitudes)."""
    g = load_golden(name)
    args = (g["object"], g["mask"], g["transfer_1"], g["transfer_2"], g["shifts"], int(g["downsample"]),
            g["measured"], float(g["scale"]))
    loss_v, go, gm = run_sweep(*args, loss=loss)
    ref_loss, ref_go, ref_gm = O.coded_sweep(*args, fp64=False, loss=loss)
    assert abs(loss_v - float(g["loss"])) <= fp32_tol(abs(ref_loss - float(g["loss"])) / abs(float(g["loss"]))) * abs(
        float(g["loss"]))
    assert rel_l2(go, g["grad_object"]) < fp32_tol(rel_l2(ref_go, g["grad_object"]))
    assert rel_l2(gm, g["grad_mask"]) < fp32_tol(rel_l2(ref_gm, g["grad_mask"]))


@pytest.mark.parametrize("nearfield,loss", [(False, "fd-isotropic"), (True, "fd-anisotropic")])
def test_fd_loss_vs_oracle_and_autograd(nearfield, loss):
    """A 128^2 field, 6 shifts, ds 2: the fd-loss sweep against the FP64 oracle, and the
    autograd entry point (ptychoX_coded_loss / ptychoX_nearfield_loss) against the sweep."""
    from ptychox_b200 import ptychoX_coded_loss, ptychoX_nearfield_loss

    obj, mask, t1, t2, shifts, meas, scale = coded_problem(128, 6, 8.0, 2, 500.0, seed=21, nearfield=nearfield)
    loss_v, go, gm = run_sweep(obj, mask, t1, t2, shifts, 2, meas, scale, loss=loss)
    ref = O.coded_sweep(obj, mask, t1, t2, shifts, 2, meas, scale, loss=loss)
    ref32 = O.coded_sweep(obj, mask, t1, t2, shifts, 2, meas, scale, fp64=False, loss=loss)
    assert abs(loss_v - ref[0]) <= fp32_tol(abs(ref32[0] - ref[0]) / abs(ref[0])) * abs(ref[0])
    assert rel_l2(go, ref[1]) < fp32_tol(rel_l2(ref32[1], ref[1]))
    assert rel_l2(gm, ref[2]) < fp32_tol(rel_l2(ref32[2], ref[2]))
    o = cuda(obj).requires_grad_(True)
    m = cuda(mask).requires_grad_(True)
    sh = cuda(shifts.astype(np.float32))
    if nearfield:
        val = ptychoX_nearfield_loss(o, m, cuda(t2), sh, 2, cuda(meas), scale, loss=loss)
    else:
        val = ptychoX_coded_loss(o, m, cuda(t1), cuda(t2), sh, 2, cuda(meas), scale, loss=loss)
    val.backward()
    assert abs(float(val.item()) - loss_v) <= 1e-12 * abs(loss_v)
    assert rel_l2(o.grad.cpu().numpy(), go) < 1e-6 and rel_l2(m.grad.cpu().numpy(), gm) < 1e-6


def test_shift_gradient_golden():
    """Position refinement: dL/dshifts against autograd through the reference's torch
    formulation (coded/ops.py:157-171), with the object and mask gradients of the same sweep."""
    from ptychox_b200.coded import coded_sweep

    g = load_golden("sweep_coded_shifts_fp64.npz")
    args = (g["object"], g["mask"], g["transfer_1"], g["transfer_2"], g["shifts"], int(g["downsample"]),
            g["measured"], float(g["scale"]))
    loss, go, gm, gs = coded_sweep(cuda(g["object"]), cuda(g["mask"]), cuda(g["transfer_1"]), cuda(g["transfer_2"]),
                                   cuda(g["shifts"].astype(np.float32)), int(g["downsample"]), cuda(g["measured"]),
                                   float(g["scale"]), with_shifts=True)
    torch.cuda.synchronize()
    ref = O.coded_sweep(*args, fp64=False, with_shifts=True)
    assert abs(float(loss.item()) - float(g["loss"])) <= TOL * abs(float(g["loss"]))
    assert rel_l2(go.cpu().numpy(), g["grad_object"]) < fp32_tol(rel_l2(ref[1], g["grad_object"]))
    assert rel_l2(gm.cpu().numpy(), g["grad_mask"]) < fp32_tol(rel_l2(ref[2], g["grad_mask"]))
    assert rel_l2(gs.cpu().numpy(), g["grad_shifts"]) < fp32_tol(rel_l2(ref[3], g["grad_shifts"]))


@pytest.mark.parametrize("loss", ["mse", "fd-isotropic"])
def test_shift_gradient_autograd_and_oracle(loss):
    """128^2 field, 6 shifts, ds 2: shifts_xy.requires_grad through ptychoX_coded_loss gives
    the FP64 oracle's shift gradient (MSE and fd_loss), and leaves the other gradients as the
    sweep without shifts."""
    from ptychox_b200 import ptychoX_coded_loss

    obj, mask, t1, t2, shifts, meas, scale = coded_problem(128, 6, 8.0, 2, 500.0, seed=23, nearfield=False)
    shifts = (shifts + np.random.default_rng(1).uniform(-0.3, 0.3, shifts.shape) / 128).astype(np.float32)
    ref = O.coded_sweep(obj, mask, t1, t2, shifts, 2, meas, scale, loss=loss, with_shifts=True)
    ref32 = O.coded_sweep(obj, mask, t1, t2, shifts, 2, meas, scale, fp64=False, loss=loss, with_shifts=True)
    o = cuda(obj).requires_grad_(True)
    m = cuda(mask).requires_grad_(True)
    sh = torch.from_numpy(shifts).requires_grad_(True)  # a CPU leaf, as a training script may hold it
    val = ptychoX_coded_loss(o, m, cuda(t1), cuda(t2), sh, 2, cuda(meas), scale, loss=loss)
    val.backward()
    assert sh.grad is not None and sh.grad.dtype == torch.float32 and sh.grad.device.type == "cpu"
    assert rel_l2(sh.grad.numpy().astype(np.float64), ref[3]) < fp32_tol(rel_l2(ref32[3], ref[3]))
    assert rel_l2(o.grad.cpu().numpy(), ref[1]) < fp32_tol(rel_l2(ref32[1], ref[1]))
    assert rel_l2(m.grad.cpu().numpy(), ref[2]) < fp32_tol(rel_l2(ref32[2], ref[2]))

