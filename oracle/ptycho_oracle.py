"""CPU oracle for the ptychography forward/adjoint sweep.

TEST INFRASTRUCTURE ONLY.  This module is the checker: it is imported by
``tests/``, by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py``.  The product path in
``ptychox_b200`` never imports it and has no CPU fallback.

It restates, in numpy/scipy, the PyTorch CPU path of PtychoX
(THUHoloLab/PtychoX, ``python/ptychoX``) for the four modalities:

* conventional: ``base/ops.py:59-67`` (forward), ``base/ops.py:92-105`` (adjoint)
* Fourier (FPM): ``fpm/ops.py:180-183`` (forward), ``fpm/ops.py:209-221`` (adjoint),
  ``fpm/ops.py:102-124`` (window indexing)
* coded: ``coded/ops.py:136-171`` (forward, phase ramp); the adjoint is the
  vector-Jacobian product that torch autograd takes through that forward, written
  out step by step in the order of ``coded_kernel.cu:347-424``
* near-field: the coded operator with ``transfer_1 = 1`` (the MATLAB near-field
  sequence ``fwd_adPtychoX_nearf.cu:58-114`` without the first transfer function)
* conventional at sub-pixel positions (no reference counterpart): the integer crop of
  ``base/ops.py:61-62`` at the rounded corner, shifted by the fractional part with
  ``shift_phase_ramp`` (``coded/ops.py:157-171``), then the conventional operator

plus the amplitude-MSE data term of the training drivers
(``train_ptychography.py:555``, ``train_fpm.py:261``, ``train_coded.py:235``:
``F.mse_loss(pred, observed)``) with the observed amplitude decoded from uint16
photon counts as ``sqrt(float32(count) * float32(scale))``.

Gradients follow PyTorch's convention for complex inputs of a real loss
(``grad = dL/dRe + i dL/dIm``), which is what the reference's hand-written
backward functions return (``python/test_ops.py`` compares them with autograd).

Parity pin: ``tests/golden/*.npz`` hold outputs of the reference's own PyTorch
path, generated by ``tests/golden/make_golden.py``; ``tests/test_oracle_golden.py``
checks this module against every one of them.

Precision: every function computes in the precision of its inputs, promoted to
complex128 when ``fp64=True`` (the FP64 oracle).  With ``fp64=False`` and
complex64 inputs it mirrors the reference's complex64 CPU path (used as the
timed CPU baseline).
"""

from __future__ import annotations

import math
import os

import numpy as np
import scipy.fft as _sfft

__all__ = [
    "measured_amplitude",
    "mse_loss_and_grad",
    "fd_loss_and_grad",
    "base_forward",
    "base_backward",
    "base_sweep",
    "base_sweep_chunked",
    "subpixel_split",
    "base_subpix_forward",
    "base_subpix_backward",
    "base_subpix_sweep",
    "fpm_flat_indices",
    "fpm_forward",
    "fpm_backward",
    "fpm_sweep",
    "shift_phase_ramp",
    "coded_forward",
    "coded_backward",
    "coded_sweep",
    "coded_sweep_chunked",
    "nearfield_sweep",
    "default_workers",
    "adam_step",
]


def default_workers() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:  # pragma: no cover - non-Linux
        return max(1, os.cpu_count() or 1)


def _cdtype(fp64: bool, *arrays) -> np.dtype:
    if fp64:
        return np.dtype(np.complex128)
    return np.result_type(*[a.dtype for a in arrays], np.complex64)


def _rdtype(cdtype) -> np.dtype:
    return np.dtype(np.float64) if np.dtype(cdtype) == np.complex128 else np.dtype(np.float32)


def _fft2(x, workers):
    return _sfft.fft2(x, axes=(-2, -1), workers=workers)


def _ifft2(x, workers):
    return _sfft.ifft2(x, axes=(-2, -1), workers=workers)


def _fftshift2(x):
    return np.fft.fftshift(x, axes=(-2, -1))


def _ifftshift2(x):
    return np.fft.ifftshift(x, axes=(-2, -1))


# ----------------------------------------------------------------------------------------
# Data term
# ----------------------------------------------------------------------------------------


def measured_amplitude(measured_u16: np.ndarray, scale: float) -> np.ndarray:
    """Observed amplitude from photon counts: ``sqrt(float32(I) * float32(scale))`` in FP32.

    The training drivers fit ``F.mse_loss(pred_amp, observed_amp)``
    (``train_ptychography.py:555``) where ``observed_amp`` is an FP32 amplitude; here it
    is decoded from uint16 counts with one correctly rounded multiply and square root,
    the same two IEEE operations the CUDA epilogue performs.
    """
    counts = np.asarray(measured_u16)
    if counts.dtype != np.uint16:
        raise TypeError("measured intensities must be uint16 counts")
    return np.sqrt(counts.astype(np.float32) * np.float32(scale))


def mse_loss_and_grad(pred: np.ndarray, observed: np.ndarray, fp64: bool = True):
    """``F.mse_loss`` (mean reduction) and its gradient ``2 (pred - obs) / numel``."""
    rd = np.float64 if fp64 else np.result_type(pred.dtype, np.float32)
    diff = pred.astype(rd) - observed.astype(rd)
    numel = diff.size
    loss = float(np.sum(diff.astype(np.float64) ** 2) / numel)
    grad = (2.0 / numel) * diff
    return loss, grad.astype(rd)


def fd_loss_and_grad(pred: np.ndarray, observed: np.ndarray, isotropic: bool = True, fp64: bool = True):
    """The periodic finite-difference data loss of ``train_coded.py:101-107`` and its gradient.

    ``D = pred - observed``; ``dx = roll(D, -1, -1) - D``, ``dy = roll(D, -1, -2) - D`` (periodic
    in the last two axes); loss ``sum(sqrt(dx^2 + dy^2 + 1e-5))`` (isotropic) or
    ``sum(|dx| + |dy|)``, summed, not averaged.  Gradient w.r.t. ``pred``: every pixel enters
    its own term and those of its left and upper neighbours,
    ``g = -(ux + uy) + roll(ux, 1, -1) + roll(uy, 1, -2)`` with ``(ux, uy) = (dx, dy) / m``
    (isotropic, ``m`` the square root) or ``(sign dx, sign dy)``.
    """
    rd = np.float64 if fp64 else np.result_type(pred.dtype, np.float32).type
    d = pred.astype(rd) - observed.astype(rd)
    dx = np.roll(d, -1, axis=-1) - d
    dy = np.roll(d, -1, axis=-2) - d
    if isotropic:
        m = np.sqrt(dx * dx + dy * dy + rd(1e-5))
        loss = float(np.sum(m.astype(np.float64)))
        ux, uy = dx / m, dy / m
    else:
        loss = float(np.sum(np.abs(dx).astype(np.float64) + np.abs(dy).astype(np.float64)))
        ux, uy = np.sign(dx), np.sign(dy)
    grad = -(ux + uy) + np.roll(ux, 1, axis=-1) + np.roll(uy, 1, axis=-2)
    return loss, grad.astype(rd)


# ----------------------------------------------------------------------------------------
# Conventional ptychography
# ----------------------------------------------------------------------------------------


def base_forward(sample, probe, positions_xy, fp64: bool = True, workers: int | None = None):
    """``abs(fftshift(fft2(crop(sample) * probe)))`` — ``python/ptychoX/base/ops.py:59-67``.

    ``positions_xy`` holds zero-based ``(x, y)`` top-left corners.  Returns
    ``(amplitude, far_field_shifted, patch_stack)`` like the reference's saved tensors.
    """
    cd = _cdtype(fp64, sample, probe)
    sample = np.asarray(sample).astype(cd, copy=False)
    probe = np.asarray(probe).astype(cd, copy=False)
    ph, pw = probe.shape
    pos = np.asarray(positions_xy, dtype=np.int64).reshape(-1, 2)
    patch_stack = np.stack([sample[y : y + ph, x : x + pw] for x, y in pos.tolist()], axis=0) if len(pos) else np.zeros((0, ph, pw), cd)
    exit_wave = patch_stack * probe[None]
    far_field = _fftshift2(_fft2(exit_wave, workers))
    amplitude = np.abs(far_field)
    return amplitude, far_field, patch_stack


def base_backward(grad_output, patch_stack, probe, far_field, positions_xy, sample_shape,
                  workers: int | None = None):
    """Hand-written adjoint of the conventional operator — ``base/ops.py:92-105``.

    ``G = ifft2(ifftshift(g * F / max(|F|, eps))) * (ph * pw)``;
    ``grad_sample[window] += G * conj(probe)``; ``grad_probe += sum_b G * conj(patch_b)``.
    ``eps`` is the machine epsilon of the real dtype (``torch.finfo(...).eps``).
    """
    cd = far_field.dtype
    rd = _rdtype(cd)
    ph, pw = probe.shape
    eps = np.finfo(rd).eps
    phase = far_field / np.maximum(np.abs(far_field), eps)
    grad_far = np.asarray(grad_output).astype(rd) * phase
    grad_exit = _ifft2(_ifftshift2(grad_far), workers) * (ph * pw)
    grad_sample = np.zeros(tuple(sample_shape), dtype=cd)
    grad_probe = np.zeros_like(probe, dtype=cd)
    probe_conj = np.conj(probe).astype(cd)
    pos = np.asarray(positions_xy, dtype=np.int64).reshape(-1, 2)
    for view, (x, y) in enumerate(pos.tolist()):
        g = grad_exit[view]
        grad_sample[y : y + ph, x : x + pw] += g * probe_conj
        grad_probe += g * np.conj(patch_stack[view])
    return grad_sample, grad_probe


def base_sweep(sample, probe, positions_xy, measured_u16, scale, fp64: bool = True,
               workers: int | None = None):
    """One sweep: forward, amplitude-MSE loss against decoded counts, adjoint.

    Returns ``(loss, grad_sample, grad_probe)``; equals ``F.mse_loss(ptychoX_base(...),
    observed).backward()`` of the reference (``train_ptychography.py:549-557``).
    """
    amp, far, patches = base_forward(sample, probe, positions_xy, fp64, workers)
    observed = measured_amplitude(measured_u16, scale)
    loss, g = mse_loss_and_grad(amp, observed, fp64=True if fp64 else False)
    gs, gp = base_backward(g, patches, np.asarray(probe).astype(far.dtype), far, positions_xy,
                           np.asarray(sample).shape, workers)
    return loss, gs, gp


def base_sweep_chunked(sample, probe, positions_xy, measured_u16, scale, chunk: int = 64,
                       workers: int | None = None):
    """:func:`base_sweep` in FP64, accumulated over chunks of ``chunk`` positions.

    The same sums as the whole-batch sweep (``F.mse_loss`` over all positions, then its
    backward): the loss sums the squared residuals of every chunk over the total element
    count, each chunk's adjoint takes ``2 (A - Y) / numel_total`` and the gradients add.
    Memory stays at one chunk of FP64 far fields (config 1: 900 x 512^2 would need 3.8 GB
    per whole-batch array).
    """
    sample = np.asarray(sample)
    probe128 = np.asarray(probe).astype(np.complex128)
    pos = np.asarray(positions_xy, dtype=np.int64).reshape(-1, 2)
    meas = np.asarray(measured_u16)
    numel = float(meas.size)
    total = 0.0
    gs = np.zeros(sample.shape, np.complex128)
    gp = np.zeros(probe128.shape, np.complex128)
    for b0 in range(0, len(pos), chunk):
        sl = slice(b0, b0 + chunk)
        amp, far, patches = base_forward(sample, probe, pos[sl], True, workers)
        diff = amp - measured_amplitude(meas[sl], scale).astype(np.float64)
        total += float(np.sum(diff * diff))
        cgs, cgp = base_backward((2.0 / numel) * diff, patches, probe128, far, pos[sl], sample.shape, workers)
        gs += cgs
        gp += cgp
    return total / numel, gs, gp


# ----------------------------------------------------------------------------------------
# Conventional ptychography at sub-pixel scan positions
# ----------------------------------------------------------------------------------------
# The reference crops integer windows only (base/ops.py:61-62).  The sub-pixel operator is
# composed from its own pieces: the window at the rounded corner (the integer crop), shifted
# by the fractional part with the reference's Fourier phase ramp (shift_phase_ramp,
# coded/ops.py:157-171, with the shift in units of the patch side: a band-limited circular
# shift of the patch), then the conventional forward (base/ops.py:59-67).


def subpixel_split(positions_xy):
    """Integer window corners ``floor(p + 1/2)`` and fractional shifts ``p - corner`` (in
    [-1/2, 1/2)) of float ``(x, y)`` scan positions."""
    p = np.asarray(positions_xy, dtype=np.float64).reshape(-1, 2)
    corner = np.floor(p + 0.5)
    return corner.astype(np.int64), p - corner


def _subpix_ramp(ph, pw, frac, rd):
    """``exp(2 pi i (dx kx / pw + dy ky / ph))`` per position (the reference's shift_phase_ramp
    with shifts ``(dx / pw, dy / ph)`` in units of the patch side)."""
    shifts = np.stack([frac[:, 0] / pw, frac[:, 1] / ph], axis=1)
    return shift_phase_ramp(ph, pw, shifts, rd)


def base_subpix_forward(sample, probe, positions_xy, fp64: bool = True, workers: int | None = None):
    """``abs(fftshift(fft2(shift(crop(sample)) * probe)))`` at float positions.

    ``shift(C) = ifft2(fft2(C) exp(2 pi i (dx kx / pw + dy ky / ph)))`` samples the cropped
    window at ``r + (dx, dy)``: position ``(x, y)`` covers the object at ``(x + c, y + r)``.
    Returns ``(amplitude, far_field_shifted, shifted_patches)``.
    """
    cd = _cdtype(fp64, sample, probe)
    rd = _rdtype(cd)
    sample = np.asarray(sample).astype(cd, copy=False)
    probe = np.asarray(probe).astype(cd, copy=False)
    ph, pw = probe.shape
    corner, frac = subpixel_split(positions_xy)
    crops = (np.stack([sample[y : y + ph, x : x + pw] for x, y in corner.tolist()], axis=0) if len(corner)
             else np.zeros((0, ph, pw), cd))
    shifted = _ifft2(_fft2(crops, workers) * _subpix_ramp(ph, pw, frac, rd), workers).astype(cd, copy=False)
    far_field = _fftshift2(_fft2(shifted * probe[None], workers))
    return np.abs(far_field), far_field, shifted


def base_subpix_backward(grad_output, shifted, probe, far_field, positions_xy, sample_shape,
                         workers: int | None = None):
    """Adjoint of :func:`base_subpix_forward` (PyTorch's complex-gradient convention).

    ``G = ifft2(ifftshift(g F / max(|F|, eps))) ph pw`` as in ``base/ops.py:92-97``;
    ``grad_probe = sum_b G conj(S_b)``; the shift is unitary up to ``1/n`` scaling, so its
    adjoint is the opposite shift: ``grad_C = ifft2(fft2(G conj(probe)) conj(ramp))``,
    added into the window at the corner.
    """
    cd = far_field.dtype
    rd = _rdtype(cd)
    ph, pw = probe.shape
    eps = np.finfo(rd).eps
    phase = far_field / np.maximum(np.abs(far_field), eps)
    grad_far = np.asarray(grad_output).astype(rd) * phase
    grad_exit = _ifft2(_ifftshift2(grad_far), workers) * (ph * pw)
    grad_probe = np.sum(grad_exit * np.conj(shifted), axis=0).astype(cd)
    corner, frac = subpixel_split(positions_xy)
    grad_crop = _ifft2(_fft2(grad_exit * np.conj(probe)[None], workers) * np.conj(_subpix_ramp(ph, pw, frac, rd)),
                       workers)
    grad_sample = np.zeros(tuple(sample_shape), dtype=cd)
    for view, (x, y) in enumerate(corner.tolist()):
        grad_sample[y : y + ph, x : x + pw] += grad_crop[view]
    return grad_sample, grad_probe


def base_subpix_sweep(sample, probe, positions_xy, measured_u16, scale, fp64: bool = True,
                      workers: int | None = None, chunk: int | None = None):
    """Forward, amplitude-MSE loss against decoded counts and adjoint at float positions, the
    training step of ``train_ptychography.py:549-557`` on the sub-pixel operator.  ``chunk``
    accumulates over chunks of positions (same sums, bounded memory)."""
    pos = np.asarray(positions_xy, dtype=np.float64).reshape(-1, 2)
    meas = np.asarray(measured_u16)
    probe_c = np.asarray(probe)
    numel = float(meas.size)
    step = len(pos) if not chunk else chunk
    total = 0.0
    gs = gp = None
    for b0 in range(0, max(len(pos), 1), max(step, 1)):
        sl = slice(b0, b0 + step)
        amp, far, shifted = base_subpix_forward(sample, probe, pos[sl], fp64, workers)
        rd = np.float64 if fp64 else np.float32
        diff = amp.astype(rd) - measured_amplitude(meas[sl], scale).astype(rd)
        total += float(np.sum(diff.astype(np.float64) ** 2))
        cgs, cgp = base_subpix_backward((rd(2.0 / numel) * diff).astype(rd), shifted, probe_c.astype(far.dtype), far,
                                        pos[sl], np.asarray(sample).shape, workers)
        gs = cgs if gs is None else gs + cgs
        gp = cgp if gp is None else gp + cgp
    return total / numel, gs, gp


# ----------------------------------------------------------------------------------------
# Fourier ptychography
# ----------------------------------------------------------------------------------------


def fpm_flat_indices(object_shape, low_shape, led_indices_xy) -> np.ndarray:
    """Flat spectrum indices of each LED window — ``fpm/ops.py:113-124``.

    ``row = (led_y + r + H // 2) % H``, ``col = (led_x + c + W // 2) % W``: ``led_indices_xy``
    is the zero-based top-left of the window in the fftshifted spectrum.
    """
    oh, ow = object_shape
    lh, lw = low_shape
    led = np.asarray(led_indices_xy, dtype=np.int64).reshape(-1, 2)
    rows = np.arange(lh, dtype=np.int64)
    cols = np.arange(lw, dtype=np.int64)
    yy = (led[:, 1, None, None] + rows[None, :, None] + oh // 2) % oh
    xx = (led[:, 0, None, None] + cols[None, None, :] + ow // 2) % ow
    return yy * ow + xx


def fpm_forward(object_field, pupil, led_indices_xy, fp64: bool = True, workers: int | None = None):
    """``abs(ifft2(fftshift(gather(fft2(O)) * pupil)))`` — ``fpm/ops.py:180-183``.

    Returns ``(amplitude, image_field, sub_spectrum)``.
    """
    cd = _cdtype(fp64, object_field, pupil)
    obj = np.asarray(object_field).astype(cd, copy=False)
    pupil = np.asarray(pupil).astype(cd, copy=False)
    spectrum = _fft2(obj, workers)
    idx = fpm_flat_indices(obj.shape, pupil.shape, led_indices_xy)
    sub = spectrum.reshape(-1)[idx]
    image = _ifft2(_fftshift2(sub * pupil[None]), workers)
    return np.abs(image), image, sub


def fpm_backward(grad_output, sub_spectrum, pupil, image_field, led_indices_xy, object_shape,
                 workers: int | None = None):
    """Hand-written FPM adjoint — ``fpm/ops.py:209-221``.

    ``Gl = ifftshift(fft2(g * z / max(|z|, eps)) / (h w))``; ``grad_pupil = sum_b Gl conj(sub)``;
    ``grad_S = index_add(Gl conj(pupil))``; ``grad_O = ifft2(grad_S) * H W``.
    """
    cd = image_field.dtype
    rd = _rdtype(cd)
    lh, lw = pupil.shape
    oh, ow = object_shape
    eps = np.finfo(rd).eps
    phase = image_field / np.maximum(np.abs(image_field), eps)
    grad_image = np.asarray(grad_output).astype(rd) * phase
    grad_low = _ifftshift2(_fft2(grad_image, workers) / (lh * lw))
    grad_pupil = np.sum(grad_low * np.conj(sub_spectrum), axis=0)
    idx = fpm_flat_indices(object_shape, (lh, lw), led_indices_xy)
    grad_spec = np.zeros(oh * ow, dtype=cd)
    np.add.at(grad_spec, idx.reshape(-1), (grad_low * np.conj(pupil)[None]).reshape(-1))
    grad_object = _ifft2(grad_spec.reshape(oh, ow), workers) * (oh * ow)
    return grad_object, grad_pupil


def fpm_sweep(object_field, pupil, led_indices_xy, measured_u16, scale, fp64: bool = True,
              workers: int | None = None):
    """Forward, amplitude-MSE loss, adjoint for FPM (``train_fpm.py:255-263``)."""
    amp, image, sub = fpm_forward(object_field, pupil, led_indices_xy, fp64, workers)
    observed = measured_amplitude(measured_u16, scale)
    loss, g = mse_loss_and_grad(amp, observed, fp64=fp64)
    go, gp = fpm_backward(g, sub, np.asarray(pupil).astype(image.dtype), image, led_indices_xy,
                          np.asarray(object_field).shape, workers)
    return loss, go, gp


# ----------------------------------------------------------------------------------------
# Coded / near-field ptychography
# ----------------------------------------------------------------------------------------


def shift_phase_ramp(height: int, width: int, shifts_xy, rdtype=np.float64) -> np.ndarray:
    """``exp(2 pi i (dx kx + dy ky))`` with signed integer frequencies — ``coded/ops.py:157-171``."""
    rdtype = np.dtype(rdtype)
    fy = (np.fft.fftfreq(height, d=1.0) * height).astype(rdtype)
    fx = (np.fft.fftfreq(width, d=1.0) * width).astype(rdtype)
    yy, xx = np.meshgrid(fy, fx, indexing="ij")
    s = np.asarray(shifts_xy).astype(rdtype).reshape(-1, 2)
    arg = rdtype.type(2.0 * math.pi) * (s[:, 0, None, None] * xx[None] + s[:, 1, None, None] * yy[None])
    return np.exp(1j * arg).astype(np.complex128 if rdtype == np.float64 else np.complex64)


def coded_forward(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample,
                  fp64: bool = True, workers: int | None = None):
    """Coded forward model — ``coded/ops.py:136-154``.

    ``x = ifft2(fft2(O) T1 ramp)``; ``s = ifft2(fft2(x M) T2)``;
    ``A = sqrt(avgpool_ds(|s|^2))``.  Returns ``(object_spectrum, x_forward, sensor_field,
    amplitude)``.  ``transfer_1=None`` means the identity (near-field).
    """
    cd = _cdtype(fp64, object_field, coded_surface)
    rd = _rdtype(cd)
    obj = np.asarray(object_field).astype(cd, copy=False)
    mask = np.asarray(coded_surface).astype(cd, copy=False)
    t2 = np.asarray(transfer_2).astype(cd, copy=False)
    h, w = obj.shape
    ramp = shift_phase_ramp(h, w, shifts_xy, rd)
    spectrum = _fft2(obj, workers)
    pre = spectrum[None] * ramp if transfer_1 is None else spectrum[None] * np.asarray(transfer_1).astype(cd)[None] * ramp
    x_forward = _ifft2(pre, workers)
    sensor = _ifft2(_fft2(x_forward * mask[None], workers) * t2[None], workers)
    ds = int(downsample)
    inten = (sensor.real ** 2 + sensor.imag ** 2).astype(rd)
    b = inten.shape[0]
    pooled = inten.reshape(b, h // ds, ds, w // ds, ds).mean(axis=(2, 4))
    amplitude = np.sqrt(np.maximum(pooled, 0.0))
    return spectrum, x_forward, sensor, amplitude


def coded_backward(grad_output, x_forward, sensor_field, amplitude, coded_surface, transfer_1,
                   transfer_2, shifts_xy, downsample, workers: int | None = None, with_shifts: bool = False):
    """Adjoint of :func:`coded_forward` (what autograd computes through ``coded/ops.py:136-154``).

    Step order follows the reference's explicit CUDA adjoint (``coded_kernel.cu:347-424``):
    RMS-pool gradient ``g / (2 A) / ds^2 * 2 s``; ``g_a = ifft2(fft2(g_s) conj(T2))``;
    ``grad_mask = sum_b g_a conj(x)``; ``g_X = fft2(g_a conj(M)) / n``;
    ``grad_spectrum = sum_b g_X conj(T1 ramp)``; ``grad_O = n ifft2(grad_spectrum)``.
    """
    cd = sensor_field.dtype
    rd = _rdtype(cd)
    h, w = sensor_field.shape[-2:]
    n = h * w
    ds = int(downsample)
    mask = np.asarray(coded_surface).astype(cd, copy=False)
    t2 = np.asarray(transfer_2).astype(cd, copy=False)
    g = np.asarray(grad_output).astype(rd)
    # d sqrt(p) = g / (2 sqrt p); avg-pool spreads /ds^2; d|s|^2 = 2 s.
    scale = g / (2.0 * amplitude) / (ds * ds)
    scale_full = np.repeat(np.repeat(scale, ds, axis=-2), ds, axis=-1)
    g_s = (2.0 * scale_full) * sensor_field
    g_a = _ifft2(_fft2(g_s, workers) * np.conj(t2)[None], workers)
    grad_mask = np.sum(g_a * np.conj(x_forward), axis=0)
    g_x = g_a * np.conj(mask)[None]
    g_big_x = _fft2(g_x, workers) / n
    ramp = shift_phase_ramp(h, w, shifts_xy, rd)
    conj_pre = np.conj(ramp) if transfer_1 is None else np.conj(ramp * np.asarray(transfer_1).astype(cd)[None])
    grad_spectrum = np.sum(g_big_x * conj_pre, axis=0)
    grad_object = _ifft2(grad_spectrum, workers) * n
    if not with_shifts:
        return grad_object, grad_mask
    # Shifts (real) enter only through the ramp of u = fft2(O) T1 ramp = fft2(x_forward):
    # du/d(dx) = 2 pi i fx u, so dL/d(dx) = Re(sum conj(G_u) du/d(dx)) = -2 pi sum fx Im(conj(G_u) u)
    # with G_u = g_big_x the PyTorch-convention gradient of u (coded/ops.py:157-171 autograd).
    u = _fft2(x_forward, workers)
    z = np.imag(np.conj(g_big_x) * u).astype(np.float64)
    fy = np.fft.fftfreq(h, d=1.0) * h
    fx = np.fft.fftfreq(w, d=1.0) * w
    gx = -2.0 * math.pi * np.einsum("bij,j->b", z, fx)
    gy = -2.0 * math.pi * np.einsum("bij,i->b", z, fy)
    return grad_object, grad_mask, np.stack([gx, gy], axis=1)


def coded_sweep(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample,
                measured_u16, scale, fp64: bool = True, workers: int | None = None, loss: str = "mse",
                with_shifts: bool = False):
    """Forward, data loss, adjoint for coded ptychography (``train_coded.py:225-237``).

    ``loss``: ``"mse"`` (``F.mse_loss``), ``"fd-isotropic"`` or ``"fd-anisotropic"``
    (``fd_loss``, ``train_coded.py:101-107``).  ``with_shifts``: also return the gradient
    w.r.t. ``shifts_xy`` ([batch, 2], what autograd gives through ``coded/ops.py:157-171``)."""
    _, xf, sensor, amp = coded_forward(object_field, coded_surface, transfer_1, transfer_2,
                                       shifts_xy, downsample, fp64, workers)
    observed = measured_amplitude(measured_u16, scale)
    if loss == "mse":
        loss, g = mse_loss_and_grad(amp, observed, fp64=fp64)
    elif loss in ("fd-isotropic", "fd-anisotropic"):
        loss, g = fd_loss_and_grad(amp, observed, isotropic=loss == "fd-isotropic", fp64=fp64)
    else:
        raise ValueError(f"unknown loss {loss!r}")
    out = coded_backward(g, xf, sensor, amp, coded_surface, transfer_1, transfer_2, shifts_xy,
                         downsample, workers, with_shifts=with_shifts)
    return (loss, *out)


def coded_sweep_chunked(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample,
                        measured_u16, scale, chunk: int = 8, fp64: bool = True, workers: int | None = None):
    """:func:`coded_sweep` (MSE) accumulated over chunks of ``chunk`` shifts.

    Each chunk's adjoint takes ``2 (A - Y) / numel_total``; the object and mask gradients are
    linear in it, so the chunks' gradients add to the whole-batch result.  ``transfer_1=None``
    gives the near-field operator.  Memory: one chunk of fields (config 3 holds 64 shifts
    of 1024^2, 1 GB per whole-batch complex128 array).  ``fp64=False`` runs the complex64
    formulation (the reference's own FP32 arithmetic) chunk by chunk.
    """
    shifts = np.asarray(shifts_xy).reshape(-1, 2)
    meas = np.asarray(measured_u16)
    numel = float(meas.size)
    rd = np.float64 if fp64 else np.float32
    total = 0.0
    go = None
    gm = None
    for b0 in range(0, len(shifts), chunk):
        sl = slice(b0, b0 + chunk)
        _, xf, sensor, amp = coded_forward(object_field, coded_surface, transfer_1, transfer_2, shifts[sl],
                                           downsample, fp64, workers)
        diff = amp.astype(rd) - measured_amplitude(meas[sl], scale).astype(rd)
        total += float(np.sum(diff.astype(np.float64) ** 2))
        cgo, cgm = coded_backward((rd(2.0 / numel) * diff).astype(rd), xf, sensor, amp, coded_surface, transfer_1,
                                  transfer_2, shifts[sl], downsample, workers)
        go = cgo if go is None else go + cgo
        gm = cgm if gm is None else gm + cgm
    return total / numel, go, gm


def nearfield_sweep(object_field, probe_field, transfer, shifts_xy, downsample, measured_u16, scale,
                    fp64: bool = True, workers: int | None = None, loss: str = "mse"):
    """Near-field = coded with ``transfer_1 = 1`` (``adPtychoX_nearf.m:44-62``)."""
    return coded_sweep(object_field, probe_field, None, transfer, shifts_xy, downsample,
                       measured_u16, scale, fp64, workers, loss)


# ----------------------------------------------------------------------------------------
# Optimiser step
# ----------------------------------------------------------------------------------------


def adam_step(param, grad, exp_avg, exp_avg_sq, step, lr, beta1=0.9, beta2=0.999, eps=1e-16,
              constraint=None):
    """One Adam step on a complex parameter, as torch.optim.Adam does it (torch/optim/adam.py,
    single-tensor path): complex values are (re, im) pairs of independent reals.

    Used by ``train_ptychography.py:500-507`` (betas (0.9, 0.999), eps 1e-16).  Optional
    projection afterwards: ``"unit_amplitude"`` (|z| <= 1, phase kept) or
    ``"real_nonnegative"`` (z -> max(Re z, 0), ``train_coded.py:242-244``).
    Returns new ``(param, exp_avg, exp_avg_sq)``; ``step`` is the 1-based step number.
    """
    rd = np.float32 if np.asarray(param).dtype == np.complex64 else np.float64
    p = np.asarray(param).view(rd).copy()
    g = np.asarray(grad).astype(param.dtype).view(rd)
    m = np.asarray(exp_avg).view(rd).copy()
    v = np.asarray(exp_avg_sq).view(rd).copy()
    m = m + rd(1 - beta1) * (g - m)
    v = rd(beta2) * v + rd(1 - beta2) * g * g
    bc1 = 1 - beta1 ** step
    bc2 = 1 - beta2 ** step
    step_size = rd(lr / bc1)
    denom = np.sqrt(v) / rd(bc2 ** 0.5) + rd(eps)
    p = p - step_size * (m / denom)
    z = p.view(np.asarray(param).dtype)
    if constraint == "unit_amplitude":
        a = np.abs(z)
        z = np.where(a > 1, z / np.maximum(a, 1e-30), z)
    elif constraint == "real_nonnegative":
        z = np.maximum(z.real, 0).astype(z.dtype)
    return z.astype(np.asarray(param).dtype), m.view(np.asarray(param).dtype), v.view(np.asarray(param).dtype)
