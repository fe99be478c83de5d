"""Conventional ptychography operator on the sm_100a library.

Drop-in for ``python/ptychoX/base/ops.py``: ``ptychoX_base`` / ``ptychography_base`` keep
the reference signature (:14-28) and the ``autograd.Function`` contract (forward saves
what backward needs, backward returns one gradient per input, :41-107).  Differences by
design: the only implementation is the CUDA library (``use_cuda_kernels`` is accepted
and ignored), and windows leaving the sample raise ``ValueError``.

``ptychoX_base_loss`` is the fused sweep: forward, amplitude-MSE against uint16 counts
and adjoint in one library call, returned as a differentiable FP64 scalar.
"""

from __future__ import annotations

import torch

from . import _abi, _status
from ._utils import (
    as_u16,
    check_complex_scan_inputs,
    device_positions,
    device_positions_subpixel,
    ptr,
    require_cuda_complex64,
    stream_handle,
    workspace,
)

__all__ = [
    "ptychoX_base",
    "ptychography_base",
    "ptychoX_base_loss",
    "ptychoX_base_subpixel",
    "ptychoX_base_subpixel_loss",
    "clear_cuda_plan_cache",
    "PtychoXBaseFunction",
    "PtychoXBaseLossFunction",
]


def ptychoX_base(
    sample: torch.Tensor,
    probe: torch.Tensor,
    positions_xy: torch.Tensor,
    use_cuda_kernels: bool = False,
) -> torch.Tensor:
    """Return ``abs(fftshift(fft2(crop(sample) * probe)))``.

    Args:
        sample: complex object tensor, shape ``[sample_h, sample_w]``.
        probe: complex probe tensor, shape ``[probe_h, probe_w]``.
        positions_xy: zero-based ``(x, y)`` scan positions, shape ``[batch, 2]``.
        use_cuda_kernels: accepted for compatibility; the sm_100a path always runs.
    """
    return PtychoXBaseFunction.apply(sample, probe, positions_xy, use_cuda_kernels)


ptychography_base = ptychoX_base


def clear_cuda_plan_cache() -> None:
    _abi.call("ptx_clear_cache")


def _prepare(sample, probe, positions_xy):
    """Validated inputs and whether the window check falls to the device (positions that
    arrive on the device, outside the ``"host"`` bounds-check mode)."""
    check_complex_scan_inputs(sample, probe, positions_xy)
    require_cuda_complex64(("sample", sample), ("probe", probe))
    sample = sample.contiguous()
    probe = probe.contiguous()
    _status.before_call(sample.device)
    pos = device_positions(positions_xy, sample.device, tuple(probe.shape), tuple(sample.shape))
    track = positions_xy.device.type != "cpu" and _status.bounds_check_mode() != "host"
    return sample, probe, pos, track


class PtychoXBaseFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sample, probe, positions_xy, use_cuda_kernels=False):  # type: ignore[override]
        sample, probe, pos, track = _prepare(sample, probe, positions_xy)
        dev = sample.device
        batch = pos.shape[0]
        ph, pw = probe.shape
        far = torch.empty((batch, ph, pw), dtype=torch.complex64, device=dev)
        amp = torch.empty((batch, ph, pw), dtype=torch.float32, device=dev)
        ws_bytes = _abi.query("ptx_base_workspace_bytes", ph, pw, batch)
        ws = workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_base_forward", ptr(sample), sample.shape[0], sample.shape[1], ptr(probe), ph, pw,
                      ptr(pos), batch, ptr(far), ptr(amp), ptr(ws), ws_bytes, stream_handle(dev))
            if track and batch:
                _status.after_call(ws, dev, "ptychoX_base")
        ctx.save_for_backward(sample, probe, far, pos)
        return amp

    @staticmethod
    def backward(ctx, grad_output):  # type: ignore[override]
        sample, probe, far, pos = ctx.saved_tensors
        dev = sample.device
        batch = pos.shape[0]
        ph, pw = probe.shape
        grad_output = grad_output.to(dtype=torch.float32).contiguous()
        grad_sample = torch.empty_like(sample)
        grad_probe = torch.empty_like(probe)
        ws_bytes = _abi.query("ptx_base_workspace_bytes", ph, pw, batch)
        ws = workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_base_backward", ptr(grad_output), ptr(far), ptr(sample), sample.shape[0],
                      sample.shape[1], ptr(probe), ph, pw, ptr(pos), batch, ptr(grad_sample), ptr(grad_probe),
                      ptr(ws), ws_bytes, stream_handle(dev))
        return grad_sample, grad_probe, None, None


SMALL_FRAMES = (32, 64, 128)
# 128^2 frames take the one-CTA-per-frame sweep only from this many frames up: that kernel
# costs about one CTA's latency per wave of frames (~30 us on a B200), the three passes
# ~11 us + 0.21 us per frame (36 frames: 18.5 against 30.5 us; 121: 36.3 against 31.9 us)
SMALL_128_MIN_FRAMES = 96


def use_small_sweep(ph: int, pw: int, batch: int) -> bool:
    """Whether a conventional sweep runs ``ptx_base_sweep_small`` (one CTA per frame)."""
    return ph == pw and pw in SMALL_FRAMES and (pw < 128 or batch >= SMALL_128_MIN_FRAMES)


def base_sweep(sample, probe, positions, measured, scale, ws=None):
    """Run one fused sweep on validated device tensors; returns ``(loss, grad_sample, grad_probe)``.

    ``positions`` must already be int64 on the device and inside the sample; ``measured``
    uint16 ``[batch, ph, pw]`` in the fftshifted layout of the forward output.
    """
    dev = sample.device
    batch = positions.shape[0]
    ph, pw = probe.shape
    loss = torch.empty((), dtype=torch.float64, device=dev)
    gs = torch.empty_like(sample)
    gp = torch.empty_like(probe)
    if ws is None:
        ws = workspace(_abi.query("ptx_base_workspace_bytes", ph, pw, batch), dev)
    # square 32 / 64 / 128 probes: the one-CTA-per-frame sweep (frame resident in shared memory)
    entry = "ptx_base_sweep_small" if use_small_sweep(ph, pw, batch) else "ptx_base_sweep"
    with torch.cuda.device(dev):
        _abi.call(entry, ptr(sample), sample.shape[0], sample.shape[1], ptr(probe), ph, pw,
                  ptr(positions), batch, ptr(measured), float(scale), ptr(loss), ptr(gs), ptr(gp), ptr(ws),
                  ws.numel(), stream_handle(dev))
    return loss, gs, gp


class PtychoXBaseLossFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sample, probe, positions_xy, measured, scale):  # type: ignore[override]
        sample, probe, pos, track = _prepare(sample, probe, positions_xy)
        meas = as_u16(measured, sample.device)
        if tuple(meas.shape) != (pos.shape[0], probe.shape[0], probe.shape[1]):
            raise ValueError("measured must have shape [batch, probe_h, probe_w].")
        dev = sample.device
        ws = workspace(_abi.query("ptx_base_workspace_bytes", probe.shape[0], probe.shape[1], pos.shape[0]), dev)
        loss, gs, gp = base_sweep(sample, probe, pos, meas, scale, ws=ws)
        if track and pos.shape[0]:
            with torch.cuda.device(dev):
                _status.after_call(ws, dev, "ptychoX_base_loss")
        ctx.save_for_backward(gs, gp)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):  # type: ignore[override]
        gs, gp = ctx.saved_tensors
        g = grad_loss.to(torch.float32)
        return gs * g, gp * g, None, None, None


def ptychoX_base_loss(
    sample: torch.Tensor,
    probe: torch.Tensor,
    positions_xy: torch.Tensor,
    measured: torch.Tensor,
    scale: float,
) -> torch.Tensor:
    """Fused ``F.mse_loss(ptychoX_base(sample, probe, positions), sqrt(scale * measured))``.

    ``measured`` holds uint16 photon counts ``[batch, ph, pw]`` in the fftshifted layout
    of ``ptychoX_base``'s output.  Returns an FP64 scalar; ``.backward()`` gives
    ``sample.grad`` / ``probe.grad`` exactly as the unfused composition does.
    """
    return PtychoXBaseLossFunction.apply(sample, probe, positions_xy, measured, scale)


# ---------------------------------------------------------------------------------------
# Sub-pixel scan positions (no reference counterpart: the reference crops integer windows,
# base/ops.py:61-62).  A float position (x, y) takes the window at floor(p + 1/2) and shifts
# it by the fraction with the reference's Fourier phase ramp (coded/ops.py:157-171).
# ---------------------------------------------------------------------------------------


def _prepare_subpixel(sample, probe, positions_xy):
    check_complex_scan_inputs(sample, probe, positions_xy)
    require_cuda_complex64(("sample", sample), ("probe", probe))
    sample = sample.contiguous()
    probe = probe.contiguous()
    _status.before_call(sample.device)
    pos = device_positions_subpixel(positions_xy, sample.device, tuple(probe.shape), tuple(sample.shape))
    track = positions_xy.device.type != "cpu" and _status.bounds_check_mode() != "host"
    return sample, probe, pos, track


def _subpixel_ws_bytes(ph, pw, batch):
    n = _abi.query("ptx_base_subpix_workspace_bytes", ph, pw, batch)
    if n == 0:
        raise ValueError(f"sub-pixel scans take probe sides that are 2^a 3^b 5^c in [16, 1024] (got {ph}x{pw}).")
    return n


def base_subpixel_sweep(sample, probe, positions, measured, scale, ws=None):
    """One fused sub-pixel sweep on validated device tensors (``positions`` float64 on the
    device); returns ``(loss, grad_sample, grad_probe)``."""
    dev = sample.device
    batch = positions.shape[0]
    ph, pw = probe.shape
    loss = torch.empty((), dtype=torch.float64, device=dev)
    gs = torch.empty_like(sample)
    gp = torch.empty_like(probe)
    if ws is None:
        ws = workspace(_subpixel_ws_bytes(ph, pw, batch), dev)
    with torch.cuda.device(dev):
        _abi.call("ptx_base_subpix_sweep", ptr(sample), sample.shape[0], sample.shape[1], ptr(probe), ph, pw,
                  ptr(positions), batch, ptr(measured), float(scale), ptr(loss), ptr(gs), ptr(gp), ptr(ws), ws.numel(),
                  stream_handle(dev))
    return loss, gs, gp


class PtychoXBaseSubpixelFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sample, probe, positions_xy):  # type: ignore[override]
        sample, probe, pos, track = _prepare_subpixel(sample, probe, positions_xy)
        dev = sample.device
        batch = pos.shape[0]
        ph, pw = probe.shape
        far = torch.empty((batch, ph, pw), dtype=torch.complex64, device=dev)
        amp = torch.empty((batch, ph, pw), dtype=torch.float32, device=dev)
        ws_bytes = _subpixel_ws_bytes(ph, pw, batch)
        ws = workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_base_subpix_forward", ptr(sample), sample.shape[0], sample.shape[1], ptr(probe), ph, pw,
                      ptr(pos), batch, ptr(far), ptr(amp), ptr(ws), ws_bytes, stream_handle(dev))
            if track and batch:
                _status.after_call(ws, dev, "ptychoX_base_subpixel")
        ctx.save_for_backward(sample, probe, far, pos)
        return amp

    @staticmethod
    def backward(ctx, grad_output):  # type: ignore[override]
        sample, probe, far, pos = ctx.saved_tensors
        dev = sample.device
        batch = pos.shape[0]
        ph, pw = probe.shape
        grad_output = grad_output.to(dtype=torch.float32).contiguous()
        grad_sample = torch.empty_like(sample)
        grad_probe = torch.empty_like(probe)
        ws_bytes = _subpixel_ws_bytes(ph, pw, batch)
        ws = workspace(ws_bytes, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_base_subpix_backward", ptr(grad_output), ptr(far), ptr(sample), sample.shape[0],
                      sample.shape[1], ptr(probe), ph, pw, ptr(pos), batch, ptr(grad_sample), ptr(grad_probe),
                      ptr(ws), ws_bytes, stream_handle(dev))
        return grad_sample, grad_probe, None


class PtychoXBaseSubpixelLossFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sample, probe, positions_xy, measured, scale):  # type: ignore[override]
        sample, probe, pos, track = _prepare_subpixel(sample, probe, positions_xy)
        meas = as_u16(measured, sample.device)
        ph, pw = probe.shape
        if tuple(meas.shape) != (pos.shape[0], ph, pw):
            raise ValueError("measured must have shape [batch, probe_h, probe_w].")
        dev = sample.device
        ws = workspace(_subpixel_ws_bytes(ph, pw, pos.shape[0]), dev)
        loss, gs, gp = base_subpixel_sweep(sample, probe, pos, meas, scale, ws=ws)
        if track and pos.shape[0]:
            with torch.cuda.device(dev):
                _status.after_call(ws, dev, "ptychoX_base_subpixel_loss")
        ctx.save_for_backward(gs, gp)
        return loss

    @staticmethod
    def backward(ctx, grad_loss):  # type: ignore[override]
        gs, gp = ctx.saved_tensors
        g = grad_loss.to(torch.float32)
        return gs * g, gp * g, None, None, None


def ptychoX_base_subpixel(sample: torch.Tensor, probe: torch.Tensor, positions_xy: torch.Tensor) -> torch.Tensor:
    """``abs(fftshift(fft2(shift(crop(sample)) * probe)))`` at float scan positions.

    ``positions_xy``: ``[batch, 2]`` zero-based ``(x, y)``, any real dtype (kept in float64).
    Each frame crops the window at ``floor(p + 1/2)`` and shifts it by the fractional part
    with a Fourier phase ramp (the reference's ``shift_phase_ramp``, ``coded/ops.py:157-171``,
    applied to the patch), so ``(x, y)`` samples the object at ``(x + c, y + r)``.  At
    integer positions this is :func:`ptychoX_base`.  Probe sides: 2^a 3^b 5^c in [16, 1024].
    Differentiable in ``sample`` and ``probe``.
    """
    return PtychoXBaseSubpixelFunction.apply(sample, probe, positions_xy)


def ptychoX_base_subpixel_loss(sample: torch.Tensor, probe: torch.Tensor, positions_xy: torch.Tensor,
                               measured: torch.Tensor, scale: float) -> torch.Tensor:
    """Fused ``F.mse_loss(ptychoX_base_subpixel(sample, probe, positions), sqrt(scale * measured))``:
    one five-pass sweep, an FP64 scalar whose ``.backward()`` fills ``sample.grad`` and
    ``probe.grad``."""
    return PtychoXBaseSubpixelLossFunction.apply(sample, probe, positions_xy, measured, scale)
