"""Fourier ptychography operator on the sm_100a library.

Drop-in for ``python/ptychoX/fpm/ops.py``: ``ptychoX_fourier`` / ``fourier_ptychography``
keep the reference signature (:14-25) and ``autograd.Function`` contract (:37-99).  The
forward saves the object spectrum ``fft2(O)`` (``[H, W]``) instead of the reference's
``[B, h, w]`` sub-spectrum stack; the backward re-gathers the windows from it.  Sides are
2^a 3^b 5^c in [4, 1024] (the reference's cuFFT takes any side; other lengths raise
``ValueError``).  ``ptychoX_fourier_loss`` is the fused sweep.
"""

from __future__ import annotations

import torch

from . import _abi
from ._utils import (as_u16, check_complex_scan_inputs, ptr, require_cuda_complex64, stream_handle, upload_small,
                     workspace)

__all__ = [
    "ptychoX_fourier",
    "fourier_ptychography",
    "ptychoX_fourier_loss",
    "clear_cuda_plan_cache",
    "PtychoXFPMFunction",
    "PtychoXFPMLossFunction",
    "fpm_sweep",
]


def ptychoX_fourier(
    object_field: torch.Tensor,
    pupil: torch.Tensor,
    led_indices_xy: torch.Tensor,
    use_cuda_kernels: bool = False,
) -> torch.Tensor:
    """Fourier ptychography amplitude operator.

    The PyTorch convention is row-major and zero-based:
    ``led_indices_xy[:, 0]`` is x and ``led_indices_xy[:, 1]`` is y (top-left corner of the
    window in the fftshifted object spectrum).
    """
    return PtychoXFPMFunction.apply(object_field, pupil, led_indices_xy, use_cuda_kernels)


fourier_ptychography = ptychoX_fourier


def clear_cuda_plan_cache() -> None:
    _abi.call("ptx_clear_cache")


def _prepare(object_field, pupil, led_indices_xy):
    check_complex_scan_inputs(object_field, pupil, led_indices_xy, "object_field", "pupil")
    require_cuda_complex64(("object_field", object_field), ("pupil", pupil))
    led = upload_small(led_indices_xy, object_field.device, torch.long)
    return object_field.contiguous(), pupil.contiguous(), led


def _ws(oh, ow, lh, lw, batch, dev):
    n = _abi.query("ptx_fpm_workspace_bytes", oh, ow, lh, lw, batch)
    return workspace(n, dev), n


class PtychoXFPMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, object_field, pupil, led_indices_xy, use_cuda_kernels=False):  # type: ignore[override]
        obj, pupil, led = _prepare(object_field, pupil, led_indices_xy)
        dev = obj.device
        (oh, ow), (lh, lw), batch = obj.shape, pupil.shape, led.shape[0]
        spectrum = torch.empty_like(obj)
        image = torch.empty((batch, lh, lw), dtype=torch.complex64, device=dev)
        amp = torch.empty((batch, lh, lw), dtype=torch.float32, device=dev)
        ws, n = _ws(oh, ow, lh, lw, batch, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_fpm_forward", ptr(obj), oh, ow, ptr(pupil), lh, lw, ptr(led), batch, ptr(spectrum),
                      ptr(image), ptr(amp), ptr(ws), n, stream_handle(dev))
        ctx.save_for_backward(spectrum, pupil, image, led)
        return amp

    @staticmethod
    def backward(ctx, grad_output):  # type: ignore[override]
        spectrum, pupil, image, led = ctx.saved_tensors
        dev = spectrum.device
        (oh, ow), (lh, lw), batch = spectrum.shape, pupil.shape, led.shape[0]
        grad_output = grad_output.to(dtype=torch.float32).contiguous()
        grad_object = torch.empty_like(spectrum)
        grad_pupil = torch.empty_like(pupil)
        ws, n = _ws(oh, ow, lh, lw, batch, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_fpm_backward", ptr(grad_output), ptr(image), ptr(spectrum), oh, ow, ptr(pupil), lh, lw,
                      ptr(led), batch, ptr(grad_object), ptr(grad_pupil), ptr(ws), n, stream_handle(dev))
        return grad_object, grad_pupil, None, None


def fpm_sweep(obj, pupil, led, measured, scale, ws=None):
    """One fused FPM sweep on device tensors; returns ``(loss, grad_object, grad_pupil)``."""
    dev = obj.device
    (oh, ow), (lh, lw), batch = obj.shape, pupil.shape, led.shape[0]
    loss = torch.empty((), dtype=torch.float64, device=dev)
    go = torch.empty_like(obj)
    gp = torch.empty_like(pupil)
    if ws is None:
        ws, _ = _ws(oh, ow, lh, lw, batch, dev)
    with torch.cuda.device(dev):
        _abi.call("ptx_fpm_sweep", ptr(obj), oh, ow, ptr(pupil), lh, lw, ptr(led), batch, ptr(measured),
                  float(scale), ptr(loss), ptr(go), ptr(gp), ptr(ws), ws.numel(), stream_handle(dev))
    return loss, go, gp


class PtychoXFPMLossFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, object_field, pupil, led_indices_xy, measured, scale):  # type: ignore[override]
        obj, pupil, led = _prepare(object_field, pupil, led_indices_xy)
        meas = as_u16(measured, obj.device)
        if tuple(meas.shape) != (led.shape[0], pupil.shape[0], pupil.shape[1]):
            raise ValueError("measured must have shape [batch, low_h, low_w].")
        loss, go, gp = fpm_sweep(obj, pupil, led, meas, scale)
        ctx.save_for_backward(go, gp)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):  # type: ignore[override]
        go, gp = ctx.saved_tensors
        g = grad_loss.to(torch.float32)
        return go * g, gp * g, None, None, None


def ptychoX_fourier_loss(object_field, pupil, led_indices_xy, measured, scale) -> torch.Tensor:
    """Fused ``F.mse_loss(ptychoX_fourier(...), sqrt(scale * measured))`` as an FP64 scalar."""
    return PtychoXFPMLossFunction.apply(object_field, pupil, led_indices_xy, measured, scale)
