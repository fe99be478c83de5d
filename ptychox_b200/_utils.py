"""Host-side input handling shared by the operators.

Mirrors ``python/ptychoX/_utils.py`` of the reference (same checks, messages and
exception types, ``check_complex_scan_inputs`` :24-42, ``matlab_positions_to_torch``
:99-101) plus what the device path needs: complex64 CUDA tensors, int64 device positions
validated against the object bounds, stream and workspace plumbing.
"""

from __future__ import annotations

import torch

from . import _abi


def check_complex_scan_inputs(
    first: torch.Tensor,
    second: torch.Tensor,
    positions_xy: torch.Tensor,
    first_name: str = "sample",
    second_name: str = "probe",
) -> None:
    """Same checks, messages and exception types as the reference (``_utils.py:24-42``)."""
    if first.ndim != 2 or second.ndim != 2:
        raise ValueError(f"{first_name} and {second_name} must be 2D complex tensors.")
    if not first.is_complex() or not second.is_complex():
        raise TypeError(f"{first_name} and {second_name} must be complex tensors.")
    if first.device != second.device:
        raise ValueError(f"{first_name} and {second_name} must live on the same device.")
    if first.dtype != second.dtype:
        raise ValueError(f"{first_name} and {second_name} must have the same dtype.")
    if positions_xy.ndim != 2 or positions_xy.shape[-1] != 2:
        raise ValueError("positions_xy must have shape [batch, 2].")
    if positions_xy.device.type != "cpu" and positions_xy.device != first.device:
        raise ValueError(f"positions_xy must be on CPU or on the same device as {first_name}.")


def require_cuda_complex64(*named: tuple[str, torch.Tensor]) -> None:
    """The sm_100a path is the only implementation: tensors must be CUDA complex64."""
    for name, t in named:
        if not t.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor (ptychox_b200 has no CPU path).")
        if t.dtype != torch.complex64:
            raise TypeError(f"{name} must be complex64 (got {t.dtype}).")


def matlab_positions_to_torch(positions_xy_1based: torch.Tensor) -> torch.Tensor:
    """Convert MATLAB one-based ``(x, y)`` scan positions to PyTorch zero-based."""
    return positions_xy_1based.to(torch.long) - 1


def device_positions(
    positions_xy: torch.Tensor,
    device: torch.device,
    window_hw: tuple[int, int],
    field_hw: tuple[int, int],
    name: str = "positions_xy",
    check_bounds: bool = True,
) -> torch.Tensor:
    """int64 contiguous positions on ``device``; windows must lie inside the field.

    The reference reads out of bounds for such windows; here they raise ``ValueError``.
    Host positions are checked on the host before the launch.  Device positions are checked
    by the kernels themselves and reported through the workspace status word
    (``_status``: deferred by default, no host synchronisation); only in the ``"host"``
    bounds-check mode are they copied to the host and checked here.
    """
    from . import _status

    pos = positions_xy.to(dtype=torch.long)
    on_host = pos.device.type == "cpu"
    if check_bounds and pos.numel() and (on_host or _status.bounds_check_mode() == "host"):
        host = pos.detach() if on_host else pos.detach().cpu()
        wh, ww = window_hw
        fh, fw = field_hw
        x, y = host[:, 0], host[:, 1]
        if bool((x < 0).any() or (y < 0).any() or (x + ww > fw).any() or (y + wh > fh).any()):
            raise ValueError(f"{name}: a {wh}x{ww} window leaves the {fh}x{fw} field.")
    return upload_small(pos, device, torch.long)


def device_positions_subpixel(
    positions_xy: torch.Tensor,
    device: torch.device,
    window_hw: tuple[int, int],
    field_hw: tuple[int, int],
    name: str = "positions_xy",
) -> torch.Tensor:
    """float64 contiguous sub-pixel positions on ``device``.  Each window starts at the rounded
    corner ``floor(p + 1/2)``; host positions are checked here as in :func:`device_positions`,
    device positions by the kernels (the workspace status word)."""
    from . import _status

    pos = positions_xy.to(dtype=torch.float64)
    on_host = pos.device.type == "cpu"
    if pos.numel() and (on_host or _status.bounds_check_mode() == "host"):
        host = pos.detach() if on_host else pos.detach().cpu()
        if not bool(torch.isfinite(host).all()):
            raise ValueError(f"{name} must be finite.")
        corner = torch.floor(host + 0.5)
        wh, ww = window_hw
        fh, fw = field_hw
        x, y = corner[:, 0], corner[:, 1]
        if bool((x < 0).any() or (y < 0).any() or (x + ww > fw).any() or (y + wh > fh).any()):
            raise ValueError(f"{name}: a {wh}x{ww} window leaves the {fh}x{fw} field.")
    return upload_small(pos, device, torch.float64)


def upload_small(t: torch.Tensor, device: torch.device, dtype: torch.dtype) -> torch.Tensor:
    """``t`` as a contiguous ``dtype`` tensor on ``device``, in order on the current stream.

    A host tensor (converted to ``dtype`` on the host first) goes through
    ``ptx_stage_host_bytes``: copied into the library's page-locked ring at the call and read
    by a kernel on the stream, so a per-step scan neither waits on a copy engine behind
    another stream's large upload nor blocks the host; device tensors are converted in place.
    """
    if t.device.type != "cpu" or torch.device(device).type != "cuda":
        return t.to(device=device, dtype=dtype).contiguous()
    host = t.detach().to(dtype=dtype).contiguous()
    out = torch.empty(host.shape, dtype=dtype, device=device)
    if host.numel():
        args = (out.data_ptr(), host.data_ptr(), host.numel() * host.element_size())
        if out.device.index == torch.cuda.current_device():
            _abi.call("ptx_stage_host_bytes", *args, stream_handle(out.device))
        else:
            with torch.cuda.device(out.device):
                _abi.call("ptx_stage_host_bytes", *args, stream_handle(out.device))
    return out


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def as_u16(measured: torch.Tensor, device: torch.device) -> torch.Tensor:
    """uint16 photon counts on ``device``; other integer dtypes are range-checked."""
    if measured.dtype != torch.uint16:
        if measured.dtype.is_floating_point or measured.dtype.is_complex:
            raise TypeError("measured intensities must be integer photon counts (uint16).")
        host = measured.detach()
        if host.numel() and (int(host.min()) < 0 or int(host.max()) > 65535):
            raise ValueError("measured counts must lie in [0, 65535].")
        measured = host.to(torch.int32).to(torch.uint16)
    return measured.to(device=device).contiguous()


def load_library():
    """Load libptychox (raises when it is missing: there is no fallback)."""
    return _abi.load()
