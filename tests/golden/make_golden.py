"""Generate golden vectors from the reference PtychoX PyTorch path.

Run in a container that has the reference checkout (read-only):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/PtychoX/python

It imports ``ptychoX`` from that directory and writes ``tests/golden/*.npz``:

* ``test_ops_{base,fpm,coded}.npz`` — the three seeded cases of the reference's own
  ``python/test_ops.py:26-104`` (seed 0, complex64, same RNG draw order), with the
  reference operator's forward output and gradients of ``(out * grad).sum()``;
* ``sweep_*_fp64.npz`` — small config-shaped problems run through the reference operator
  in complex128 followed by ``F.mse_loss(pred, observed)`` and ``.backward()`` (the
  training drivers' step, ``train_ptychography.py:549-557``), with uint16 Poisson counts
  decoded as ``sqrt(float32(I) * float32(scale))``: loss and gradients;
* ``sweep_coded_fd_{iso,aniso}_fp64.npz`` — the coded problem with the reference's own
  ``fd_loss`` (``train_coded.py:101-107``, imported from the reference's ``train_coded``
  module) in place of the MSE;
* ``sweep_base_subpix_fp64.npz`` — the conventional sweep at sub-pixel (float) positions,
  composed from the reference's crop, ``shift_phase_ramp`` (``coded/ops.py:157-171``) and
  ``ptychoX_base`` (the reference has no sub-pixel operator of its own).

``REFERENCE_PYTHON_DIR`` is required; a second argument ``fd``, ``shifts`` or ``subpix``
regenerates only that family.

The fixtures are small (a few hundred KB in total) and are the parity pin of the
numpy oracle (``oracle/``) and of the CUDA library.
"""

from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import torch
import torch.nn.functional as F

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))  # repo root, for ptychox_b200.synth

from ptychox_b200 import synth  # noqa: E402


def _np(t):
    return t.detach().cpu().numpy()


def test_ops_cases(ptychoX):
    """Replicates python/test_ops.py:26-104 on CPU (use_cuda_kernels=False)."""
    torch.manual_seed(0)
    sample0 = torch.randn(9, 10, dtype=torch.complex64)
    probe0 = torch.randn(4, 5, dtype=torch.complex64)
    positions = torch.tensor([[0, 0], [2, 3], [5, 4]], dtype=torch.long)
    grad = torch.randn(3, 4, 5)
    sample = sample0.clone().requires_grad_(True)
    probe = probe0.clone().requires_grad_(True)
    out = ptychoX.ptychoX_base(sample, probe, positions)
    (out * grad).sum().backward()
    np.savez(HERE / "test_ops_base.npz", sample=_np(sample0), probe=_np(probe0), positions=_np(positions),
             grad=_np(grad), out=_np(out), grad_sample=_np(sample.grad), grad_probe=_np(probe.grad))

    object0 = torch.randn(16, 16, dtype=torch.complex64)
    pupil0 = torch.randn(8, 8, dtype=torch.complex64)
    leds = torch.tensor([[0, 0], [2, 1], [6, 5]], dtype=torch.long)
    fpm_grad = torch.randn(3, 8, 8)
    obj = object0.clone().requires_grad_(True)
    pup = pupil0.clone().requires_grad_(True)
    out = ptychoX.ptychoX_fourier(obj, pup, leds)
    (out * fpm_grad).sum().backward()
    np.savez(HERE / "test_ops_fpm.npz", object=_np(object0), pupil=_np(pupil0), leds=_np(leds), grad=_np(fpm_grad),
             out=_np(out), grad_object=_np(obj.grad), grad_pupil=_np(pup.grad))

    coded_object0 = torch.randn(16, 16, dtype=torch.complex64)
    coded_mask0 = torch.randn(16, 16, dtype=torch.complex64)
    transfer1 = torch.randn(16, 16, dtype=torch.complex64)
    transfer2 = torch.randn(16, 16, dtype=torch.complex64)
    shifts = torch.tensor([[0.01, -0.02], [0.03, 0.01]], dtype=torch.float32)
    coded_grad = torch.randn(2, 8, 8)
    co = coded_object0.clone().requires_grad_(True)
    cm = coded_mask0.clone().requires_grad_(True)
    out = ptychoX.ptychoX_coded(co, cm, transfer1, transfer2, shifts, 2)
    (out * coded_grad).sum().backward()
    np.savez(HERE / "test_ops_coded.npz", object=_np(coded_object0), mask=_np(coded_mask0),
             transfer_1=_np(transfer1), transfer_2=_np(transfer2), shifts=_np(shifts), downsample=2,
             grad=_np(coded_grad), out=_np(out), grad_object=_np(co.grad), grad_mask=_np(cm.grad))


def _observed(counts: np.ndarray, scale: float) -> torch.Tensor:
    amp32 = np.sqrt(counts.astype(np.float32) * np.float32(scale))
    return torch.from_numpy(amp32.astype(np.float64))


def _loss_step(fn, params, observed, loss_fn=None):
    leaves = [torch.from_numpy(p.astype(np.complex128)).requires_grad_(True) for p in params]
    pred = fn(*leaves)
    loss = F.mse_loss(pred, observed) if loss_fn is None else loss_fn(pred, observed)
    loss.backward()
    return float(loss.item()), [_np(x.grad) for x in leaves]


def sweep_base(ptychoX, name, n_obj, ph, pw, grid, step, origin, jitter, photons, seed):
    rng = np.random.default_rng(seed)
    obj_true = synth.random_object(n_obj, n_obj, rng)
    probe_true = synth.gaussian_probe(ph, pw, rng)
    pos = synth.raster_positions(grid, step, origin, jitter, rng)
    pos_t = torch.from_numpy(pos)
    with torch.no_grad():
        amp = ptychoX.ptychoX_base(torch.from_numpy(obj_true.astype(np.complex128)),
                                   torch.from_numpy(probe_true.astype(np.complex128)), pos_t)
    counts, scale = synth.poisson_counts(_np(amp) ** 2, photons, rng)
    # evaluate away from the truth so residuals are not pure noise
    obj = (obj_true * (1.0 + 0.15 * rng.standard_normal(obj_true.shape))).astype(np.complex64)
    probe = (probe_true * np.exp(0.2j * rng.standard_normal(probe_true.shape))).astype(np.complex64)
    loss, (g_obj, g_probe) = _loss_step(lambda o, p: ptychoX.ptychoX_base(o, p, pos_t), [obj, probe],
                                        _observed(counts, scale))
    np.savez(HERE / name, sample=obj, probe=probe, positions=pos, measured=counts, scale=np.float32(scale),
             loss=loss, grad_sample=g_obj, grad_probe=g_probe)


def sweep_base_subpix(ptychoX, name, n_obj, ph, pw, grid, step, origin, jitter, photons, seed):
    """Conventional sweep at sub-pixel positions, composed from the reference's own functions
    (it has no sub-pixel operator): the crop of base/ops.py:61-62 at the rounded corner
    floor(p + 1/2), the fractional shift by shift_phase_ramp (coded/ops.py:157-171, shifts in
    units of the patch side) applied to the patch's spectrum, and ptychoX_base on the shifted
    patch (its own sample, position (0, 0)); autograd takes the gradients through it all."""
    from ptychoX.coded.ops import shift_phase_ramp

    rng = np.random.default_rng(seed)
    obj_true = synth.random_object(n_obj, n_obj, rng)
    probe_true = synth.gaussian_probe(ph, pw, rng)
    pos = synth.raster_positions_subpixel(grid, step, origin, jitter, rng)
    corner = np.floor(pos + 0.5)
    frac = pos - corner
    shifts = torch.from_numpy(np.stack([frac[:, 0] / pw, frac[:, 1] / ph], axis=1))
    zero = torch.zeros(1, 2, dtype=torch.long)

    def forward(o, pr):
        ramp = shift_phase_ramp(ph, pw, shifts, o.device, torch.float64)
        outs = []
        for b, (x, y) in enumerate(corner.astype(np.int64).tolist()):
            crop = o[y : y + ph, x : x + pw]
            patch = torch.fft.ifft2(torch.fft.fft2(crop) * ramp[b])
            outs.append(ptychoX.ptychoX_base(patch, pr, zero))
        return torch.cat(outs, dim=0)

    with torch.no_grad():
        amp = forward(torch.from_numpy(obj_true.astype(np.complex128)), torch.from_numpy(probe_true.astype(np.complex128)))
    counts, scale = synth.poisson_counts(_np(amp) ** 2, photons, rng)
    obj = (obj_true * (1.0 + 0.15 * rng.standard_normal(obj_true.shape))).astype(np.complex64)
    probe = (probe_true * np.exp(0.2j * rng.standard_normal(probe_true.shape))).astype(np.complex64)
    loss, (g_obj, g_probe) = _loss_step(forward, [obj, probe], _observed(counts, scale))
    np.savez(HERE / name, sample=obj, probe=probe, positions=pos, measured=counts, scale=np.float32(scale),
             loss=loss, grad_sample=g_obj, grad_probe=g_probe)


def subpix_case(ptychoX):
    sweep_base_subpix(ptychoX, "sweep_base_subpix_fp64.npz", 96, 16, 32, 4, 12, 6, 2.5, 1e4, seed=17)


def sweep_fpm(ptychoX, name, n, h, leds_grid, photons, seed):
    rng = np.random.default_rng(seed)
    obj_true = synth.random_object(n, n, rng)
    pupil = synth.circular_pupil(h, 0.3)
    step = max(1, (n - h) // (leds_grid + 1))
    c = (n - h) // 2
    offs = (np.arange(leds_grid) - (leds_grid - 1) / 2.0) * step
    led = np.array([[c + int(round(x)), c + int(round(y))] for y in offs for x in offs], dtype=np.int64)
    led_t = torch.from_numpy(led)
    with torch.no_grad():
        amp = ptychoX.ptychoX_fourier(torch.from_numpy(obj_true.astype(np.complex128)),
                                      torch.from_numpy(pupil.astype(np.complex128)), led_t)
    counts, scale = synth.poisson_counts(_np(amp) ** 2, photons, rng, per_pixel=True)
    obj = (obj_true * (1.0 + 0.15 * rng.standard_normal(obj_true.shape))).astype(np.complex64)
    pup = (pupil * np.exp(0.3j * rng.standard_normal(pupil.shape))).astype(np.complex64)
    loss, (g_obj, g_pup) = _loss_step(lambda o, p: ptychoX.ptychoX_fourier(o, p, led_t), [obj, pup],
                                      _observed(counts, scale))
    np.savez(HERE / name, object=obj, pupil=pup, leds=led, measured=counts, scale=np.float32(scale), loss=loss,
             grad_object=g_obj, grad_pupil=g_pup)


def sweep_coded(ptychoX, name, n, ds, count, photons, seed, nearfield, loss_fn=None):
    rng = np.random.default_rng(seed)
    obj_true = synth.random_object(n, n, rng)
    mask = synth.binary_mask(n, 0.5, rng)
    dx = 1.85e-6
    t2 = synth.angular_spectrum_transfer(n, dx, 0.5e-6, 2e-3)
    t1 = np.ones((n, n), np.complex64) if nearfield else synth.angular_spectrum_transfer(n, dx, 0.5e-6, 396.95e-6)
    shifts = synth.coded_shifts(count, 3.0, n, rng)
    sh_t = torch.from_numpy(shifts)
    t1_t = torch.from_numpy(t1.astype(np.complex128))
    t2_t = torch.from_numpy(t2.astype(np.complex128))
    with torch.no_grad():
        amp = ptychoX.ptychoX_coded(torch.from_numpy(obj_true.astype(np.complex128)),
                                    torch.from_numpy(mask.astype(np.complex128)), t1_t, t2_t, sh_t, ds)
    counts, scale = synth.poisson_counts(_np(amp) ** 2, photons, rng, per_pixel=True)
    obj = (obj_true * (1.0 + 0.15 * rng.standard_normal(obj_true.shape))).astype(np.complex64)
    msk = (mask * (1.0 + 0.1 * rng.standard_normal(mask.shape)) + 0.05).astype(np.complex64)
    loss, (g_obj, g_mask) = _loss_step(lambda o, m: ptychoX.ptychoX_coded(o, m, t1_t, t2_t, sh_t, ds), [obj, msk],
                                       _observed(counts, scale), loss_fn)
    np.savez(HERE / name, object=obj, mask=msk, transfer_1=t1, transfer_2=t2, shifts=shifts, downsample=ds,
             measured=counts, scale=np.float32(scale), loss=loss, grad_object=g_obj, grad_mask=g_mask,
             nearfield=nearfield)


def shift_case(ptychoX):
    """Gradient w.r.t. the coded shifts: the reference's torch formulation
    (``coded/ops.py:136-171``, differentiable in ``shifts_xy`` through ``shift_phase_ramp``)
    in complex128 with the MSE loss, written with every gradient."""
    from ptychoX.coded.ops import _coded_forward_torch

    n, ds, count, photons, seed = 32, 2, 4, 200.0, 17
    rng = np.random.default_rng(seed)
    obj_true = synth.random_object(n, n, rng)
    mask = synth.binary_mask(n, 0.5, rng)
    dx = 1.85e-6
    t2 = synth.angular_spectrum_transfer(n, dx, 0.5e-6, 2e-3)
    t1 = synth.angular_spectrum_transfer(n, dx, 0.5e-6, 396.95e-6)
    shifts = synth.coded_shifts(count, 3.0, n, rng)
    t1_t = torch.from_numpy(t1.astype(np.complex128))
    t2_t = torch.from_numpy(t2.astype(np.complex128))
    with torch.no_grad():
        amp = _coded_forward_torch(torch.from_numpy(obj_true.astype(np.complex128)),
                                   torch.from_numpy(mask.astype(np.complex128)), t1_t, t2_t,
                                   torch.from_numpy(shifts.astype(np.float64)), ds)[3]
    counts, scale = synth.poisson_counts(_np(amp) ** 2, photons, rng, per_pixel=True)
    obj = (obj_true * (1.0 + 0.15 * rng.standard_normal(obj_true.shape))).astype(np.complex64)
    msk = (mask * (1.0 + 0.1 * rng.standard_normal(mask.shape)) + 0.05).astype(np.complex64)
    # evaluate with shifts off by up to 0.3 px so the shift gradient is far from zero
    sh_eval = (shifts + rng.uniform(-0.3, 0.3, shifts.shape) / n).astype(np.float32)
    o = torch.from_numpy(obj.astype(np.complex128)).requires_grad_(True)
    m = torch.from_numpy(msk.astype(np.complex128)).requires_grad_(True)
    sh = torch.from_numpy(sh_eval.astype(np.float64)).requires_grad_(True)
    pred = _coded_forward_torch(o, m, t1_t, t2_t, sh, ds)[3]
    loss = F.mse_loss(pred, _observed(counts, scale))
    loss.backward()
    np.savez(HERE / "sweep_coded_shifts_fp64.npz", object=obj, mask=msk, transfer_1=t1, transfer_2=t2,
             shifts=sh_eval, downsample=ds, measured=counts, scale=np.float32(scale), loss=float(loss.item()),
             grad_object=_np(o.grad), grad_mask=_np(m.grad), grad_shifts=_np(sh.grad))


def fd_cases(ptychoX):
    import train_coded  # the reference's coded training driver (defines fd_loss)

    for iso, tag in ((True, "iso"), (False, "aniso")):
        sweep_coded(ptychoX, f"sweep_coded_fd_{tag}_fp64.npz", 32, 2, 4, 200.0, seed=16, nearfield=False,
                    loss_fn=lambda p, o, iso=iso: train_coded.fd_loss(p, o, isotropic=iso))


def main(ref_python_dir: str) -> None:
    sys.dont_write_bytecode = True
    sys.path.insert(0, ref_python_dir)
    import ptychoX  # the reference package

    test_ops_cases(ptychoX)
    sweep_base(ptychoX, "sweep_base_fp64.npz", 64, 16, 16, 5, 10, 4, 2, 1e4, seed=11)
    sweep_base(ptychoX, "sweep_base_odd_fp64.npz", 40, 15, 12, 3, 9, 2, 1, 5e3, seed=12)
    sweep_fpm(ptychoX, "sweep_fpm_fp64.npz", 64, 16, 3, 500.0, seed=13)
    sweep_coded(ptychoX, "sweep_coded_fp64.npz", 32, 2, 4, 200.0, seed=14, nearfield=False)
    sweep_coded(ptychoX, "sweep_nearfield_fp64.npz", 32, 4, 3, 200.0, seed=15, nearfield=True)
    fd_cases(ptychoX)
    shift_case(ptychoX)
    subpix_case(ptychoX)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py REFERENCE_PYTHON_DIR [fd|shifts|subpix]")
    if len(sys.argv) > 2 and sys.argv[2] in ("fd", "shifts", "subpix"):  # one family of fixtures only
        sys.dont_write_bytecode = True
        sys.path.insert(0, sys.argv[1])
        import ptychoX  # noqa: E402

        {"fd": fd_cases, "shifts": shift_case, "subpix": subpix_case}[sys.argv[2]](ptychoX)
    else:
        main(sys.argv[1])
