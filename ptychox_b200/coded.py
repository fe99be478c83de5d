"""Coded and near-field ptychography operators on the sm_100a library.

Drop-in for ``python/ptychoX/coded/ops.py``: ``ptychoX_coded`` / ``coded_ptychography``
keep the reference signature (:22-62), input checks and messages (``_check_inputs``
:174-200) and the ``autograd.Function`` contract (:68-133, seven gradients).  The
reference differentiates its torch path with autograd when the CUDA extension is not
used; here the hand-written adjoint always runs (it equals autograd's product).

``ptychoX_nearfield(object_field, probe_field, transfer, shifts_xy, downsample)`` is the
near-field operator of the MATLAB class ``adPtychoX_nearf`` = coded with
``transfer_1 = 1``.  Fields are square with a 2^a 3^b 5^c side in [16, 1024] (the
reference's cuFFT takes any side; other sides raise ``ValueError``); ``downsample`` must
divide the side (and, for power-of-two sides, the row group of 8, for others a row group of
at most 512 threads).
"""

from __future__ import annotations

import torch

from . import _abi
from ._utils import as_u16, ptr, stream_handle, upload_small, workspace

__all__ = [
    "ptychoX_coded",
    "coded_ptychography",
    "ptychoX_nearfield",
    "nearfield_ptychography",
    "ptychoX_coded_loss",
    "ptychoX_nearfield_loss",
    "clear_cuda_plan_cache",
    "PtychoXCodedFunction",
    "coded_sweep",
]


def clear_cuda_plan_cache() -> None:
    _abi.call("ptx_clear_cache")


def _check_inputs(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample) -> None:
    """Same checks and messages as the reference (``coded/ops.py:174-200``)."""
    if object_field.ndim != 2:
        raise ValueError("object_field must be a 2D complex tensor.")
    named = [("coded_surface", coded_surface), ("transfer_2", transfer_2)]
    if transfer_1 is not None:
        named.insert(1, ("transfer_1", transfer_1))
    for name, tensor in named:
        if tensor.shape != object_field.shape:
            raise ValueError(f"{name} must have the same shape as object_field.")
        if tensor.device != object_field.device:
            raise ValueError(f"{name} must live on the same device as object_field.")
    if not object_field.is_complex() or not coded_surface.is_complex():
        raise TypeError("object_field and coded_surface must be complex tensors.")
    if (transfer_1 is not None and not transfer_1.is_complex()) or not transfer_2.is_complex():
        raise TypeError("transfer_1 and transfer_2 must be complex tensors.")
    if shifts_xy.ndim != 2 or shifts_xy.shape[-1] != 2:
        raise ValueError("shifts_xy must have shape [batch, 2].")
    if object_field.shape[0] % downsample != 0 or object_field.shape[1] % downsample != 0:
        raise ValueError("object_field shape must be divisible by downsample.")


def _prepare(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample):
    _check_inputs(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample)
    for name, t in (("object_field", object_field), ("coded_surface", coded_surface), ("transfer_2", transfer_2),
                    ("transfer_1", transfer_1)):
        if t is None:
            continue
        if not t.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor (ptychox_b200 has no CPU path).")
        if t.dtype != torch.complex64:
            raise TypeError(f"{name} must be complex64 (got {t.dtype}).")
    h, w = object_field.shape
    if h != w:
        raise ValueError("coded / near-field fields must be square.")
    dev = object_field.device
    shifts = upload_small(shifts_xy, dev, torch.float32)
    t1 = None if transfer_1 is None else transfer_1.contiguous()
    return object_field.contiguous(), coded_surface.contiguous(), t1, transfer_2.contiguous(), shifts


def _ws(n, batch, dev):
    nb = _abi.query("ptx_coded_workspace_bytes", n, batch)
    return workspace(nb, dev), nb


class PtychoXCodedFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample,  # type: ignore[override]
                use_cuda_kernels=False):
        obj, mask, t1, t2, shifts = _prepare(object_field, coded_surface, transfer_1, transfer_2, shifts_xy,
                                             downsample)
        dev = obj.device
        n, batch, ds = obj.shape[0], shifts.shape[0], int(downsample)
        xf = torch.empty((batch, n, n), dtype=torch.complex64, device=dev)
        sensor = torch.empty_like(xf)
        amp = torch.empty((batch, n // ds, n // ds), dtype=torch.float32, device=dev)
        ws, nb = _ws(n, batch, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_coded_forward", ptr(obj), ptr(mask), ptr(t1), ptr(t2), n, ptr(shifts), batch, ds,
                      ptr(xf), ptr(sensor), ptr(amp), ptr(ws), nb, stream_handle(dev))
        ctx.save_for_backward(xf, sensor, amp, mask, t2, shifts, *(() if t1 is None else (t1,)))
        ctx.downsample = ds
        ctx.has_t1 = t1 is not None
        return amp

    @staticmethod
    def backward(ctx, grad_output):  # type: ignore[override]
        saved = ctx.saved_tensors
        xf, sensor, amp, mask, t2, shifts = saved[:6]
        t1 = saved[6] if ctx.has_t1 else None
        dev = mask.device
        n, batch = mask.shape[0], shifts.shape[0]
        grad_output = grad_output.to(dtype=torch.float32).contiguous()
        grad_object = torch.empty_like(mask)
        grad_coded = torch.empty_like(mask)
        ws, nb = _ws(n, batch, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_coded_backward", ptr(grad_output), ptr(xf), ptr(sensor), ptr(amp), ptr(mask), ptr(t1),
                      ptr(t2), n, ptr(shifts), batch, ctx.downsample, ptr(grad_object), ptr(grad_coded), ptr(ws), nb,
                      stream_handle(dev))
        return grad_object, grad_coded, None, None, None, None, None


def ptychoX_coded(
    object_field: torch.Tensor,
    coded_surface: torch.Tensor,
    transfer_1: torch.Tensor,
    transfer_2: torch.Tensor,
    shifts_xy: torch.Tensor,
    downsample: int,
    use_cuda_kernels: bool = False,
) -> torch.Tensor:
    """Forward model for coded ptychography.

    Args:
        object_field: high-resolution complex object, ``[H, W]``.
        coded_surface: high-resolution complex coded surface, ``[H, W]``.
        transfer_1: propagation transfer function before the coded surface.
        transfer_2: propagation transfer function after the coded surface.
        shifts_xy: normalized subpixel shifts, ``[batch, 2]``, ``(dx, dy)``.
        downsample: integer detector downsample factor.

    Returns:
        RMS downsampled amplitudes, shape ``[batch, H/downsample, W/downsample]``.
    """
    return PtychoXCodedFunction.apply(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample,
                                      use_cuda_kernels)


coded_ptychography = ptychoX_coded


def ptychoX_nearfield(object_field, probe_field, transfer, shifts_xy, downsample) -> torch.Tensor:
    """Near-field ptychography: ``ptychoX_coded`` with ``transfer_1 = 1``.

    ``probe_field`` is the diffuser / structured illumination multiplied after the shifted
    object (the MATLAB ``adPtychoX_nearf`` "wavefront2"), ``transfer`` the propagator to
    the detector (``adPtychoX_nearf.m:44-62``).
    """
    return PtychoXCodedFunction.apply(object_field, probe_field, None, transfer, shifts_xy, downsample, True)


nearfield_ptychography = ptychoX_nearfield


LOSSES = ("mse", "fd-isotropic", "fd-anisotropic")


def coded_sweep(obj, mask, t1, t2, shifts, downsample, measured, scale, ws=None, loss="mse", with_shifts=False):
    """One fused coded (or near-field, ``t1=None``) sweep; returns ``(loss, grad_object, grad_mask)``,
    plus the FP64 gradient w.r.t. the shifts (``[batch, 2]``) when ``with_shifts``.

    ``loss``: ``"mse"`` (``F.mse_loss``) or the periodic finite-difference loss of
    ``train_coded.py:101-107`` (``"fd-isotropic"`` / ``"fd-anisotropic"``).
    """
    if loss not in LOSSES:
        raise ValueError(f"loss must be one of {LOSSES}, got {loss!r}")
    dev = obj.device
    n, batch = obj.shape[0], shifts.shape[0]
    out = torch.empty((), dtype=torch.float64, device=dev)
    go = torch.empty_like(obj)
    gm = torch.empty_like(mask)
    if with_shifts:
        kind = LOSSES.index(loss)  # PTX_LOSS_MSE / _FD_ISOTROPIC / _FD_ANISOTROPIC
        gs = torch.empty((batch, 2), dtype=torch.float64, device=dev)
        if ws is None:
            ws = workspace(_abi.query("ptx_coded_sweep_ex_workspace_bytes", n, batch, int(downsample), kind), dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_coded_sweep_ex", ptr(obj), ptr(mask), ptr(t1), ptr(t2), n, ptr(shifts), batch,
                      int(downsample), ptr(measured), float(scale), kind, ptr(out), ptr(go), ptr(gm), ptr(gs),
                      ptr(ws), ws.numel(), stream_handle(dev))
        return out, go, gm, gs
    with torch.cuda.device(dev):
        if loss == "mse":
            if ws is None:
                ws, _ = _ws(n, batch, dev)
            _abi.call("ptx_coded_sweep", ptr(obj), ptr(mask), ptr(t1), ptr(t2), n, ptr(shifts), batch,
                      int(downsample), ptr(measured), float(scale), ptr(out), ptr(go), ptr(gm), ptr(ws), ws.numel(),
                      stream_handle(dev))
        else:
            if ws is None:
                ws = workspace(_abi.query("ptx_coded_fd_workspace_bytes", n, batch, int(downsample)), dev)
            _abi.call("ptx_coded_sweep_fd", ptr(obj), ptr(mask), ptr(t1), ptr(t2), n, ptr(shifts), batch,
                      int(downsample), ptr(measured), float(scale), int(loss == "fd-isotropic"), ptr(out), ptr(go),
                      ptr(gm), ptr(ws), ws.numel(), stream_handle(dev))
    return out, go, gm


class PtychoXCodedLossFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample, measured,  # type: ignore[override]
                scale, loss="mse"):
        obj, mask, t1, t2, shifts = _prepare(object_field, coded_surface, transfer_1, transfer_2, shifts_xy,
                                             downsample)
        n, ds = obj.shape[0], int(downsample)
        meas = as_u16(measured, obj.device)
        if tuple(meas.shape) != (shifts.shape[0], n // ds, n // ds):
            raise ValueError("measured must have shape [batch, H/downsample, W/downsample].")
        ctx.shift_dtype = shifts_xy.dtype if torch.is_tensor(shifts_xy) else torch.float32
        ctx.shift_device = shifts_xy.device if torch.is_tensor(shifts_xy) else obj.device
        if ctx.needs_input_grad[4]:
            # position refinement: the shifts enter through the phase ramp only
            value, go, gm, gs = coded_sweep(obj, mask, t1, t2, shifts, ds, meas, scale, loss=loss, with_shifts=True)
            ctx.save_for_backward(go, gm, gs)
        else:
            value, go, gm = coded_sweep(obj, mask, t1, t2, shifts, ds, meas, scale, loss=loss)
            ctx.save_for_backward(go, gm)
        return value

    @staticmethod
    def backward(ctx, grad_loss):  # type: ignore[override]
        saved = ctx.saved_tensors
        go, gm = saved[0], saved[1]
        g = grad_loss.to(torch.float32)
        g_shift = None
        if len(saved) == 3:
            g_shift = (saved[2] * grad_loss.to(torch.float64)).to(device=ctx.shift_device, dtype=ctx.shift_dtype)
        return go * g, gm * g, None, None, g_shift, None, None, None, None


def ptychoX_coded_loss(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample, measured,
                       scale, loss: str = "mse") -> torch.Tensor:
    """Fused ``F.mse_loss(ptychoX_coded(...), sqrt(scale * measured))`` as an FP64 scalar;
    ``loss="fd-isotropic"`` / ``"fd-anisotropic"`` gives ``fd_loss`` (``train_coded.py:101-107``)."""
    return PtychoXCodedLossFunction.apply(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample,
                                          measured, scale, loss)


def ptychoX_nearfield_loss(object_field, probe_field, transfer, shifts_xy, downsample, measured,
                           scale, loss: str = "mse") -> torch.Tensor:
    """Fused near-field sweep (``transfer_1 = 1``) as an FP64 scalar; ``loss`` as in
    ``ptychoX_coded_loss``."""
    return PtychoXCodedLossFunction.apply(object_field, probe_field, None, transfer, shifts_xy, downsample, measured,
                                          scale, loss)
