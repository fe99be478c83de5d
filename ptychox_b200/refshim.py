"""libptychox behind the reference's own native-extension contract.

The reference's operators reach their CUDA code through a pybind11 module per modality
(``ptychoX.{base,fpm,coded}._C``), loaded by each ``ops.py``'s ``_load_cuda_ext`` into a
module-level ``_CUDA_EXT`` and called as ``_C.forward(...)`` / ``_C.backward(...)`` /
``_C.clear_plan_cache()`` (``python/ptychoX/csrc/base_extension.cpp:21-66``,
``fpm_extension.cpp:21-66``, ``coded_extension.cpp:26-94``; call sites
``base/ops.py:57,83-91``, ``fpm/ops.py:53,75-83``, ``coded/ops.py:88-95,120-130``; loaders
``base/ops.py:110-124``, ``fpm/ops.py:127-141``, ``coded/ops.py:203-217``).
``BASE``, ``FOURIER`` and ``CODED`` below keep that contract -- the same arguments, the same
return arity, CUDA / dtype checks raising ``RuntimeError`` like ``TORCH_CHECK`` -- and run on
libptychox.  :func:`install` points an imported reference package at them, so
``ptychoX_base(..., use_cuda_kernels=True)`` and its siblings run the sm_100a kernels with the
reference's own ``autograd.Function`` classes unchanged.

The saved-tensor slots keep their shapes where the reference's backward reads them and
carry what libptychox's adjoint needs:

* conventional: the ``patch_stack`` slot is a ``[batch, ph, pw]`` view of the sample (batch
  stride 0), so ``base/ops.py:78`` unpacks it; the adjoint re-reads the object patches from
  the sample it points at instead of a 1.9 GB stack (900 x 512^2).  Modifying the sample in
  place between forward and backward is therefore caught by autograd's version check;
* Fourier: the ``sub_spectrum`` slot holds the whole object spectrum ``fft2(object)``
  (``[H, W]``), which libptychox's adjoint gathers its windows from;
* coded: the ``object_spectrum`` slot holds the pooled amplitude, which libptychox's exact
  RMS-pool adjoint takes (the reference's backward passes the slot through unread).
"""

from __future__ import annotations

import torch

from . import _abi
from ._utils import ptr, stream_handle, workspace


def _check(cond: bool, msg: str) -> None:
    if not cond:
        raise RuntimeError(msg)  # TORCH_CHECK raises RuntimeError


def _cuda_dtype(t: torch.Tensor, name: str, dtype: torch.dtype, label: str) -> None:
    _check(t.is_cuda, f"{name} must be a CUDA tensor")
    _check(t.dtype == dtype, f"{name} must be {label}")


class _Base:
    """``ptychoX.base._C`` on libptychox (``base_extension.cpp:21-66``)."""

    @staticmethod
    def forward(sample: torch.Tensor, probe: torch.Tensor, positions_xy: torch.Tensor):
        _cuda_dtype(sample, "sample", torch.complex64, "complex64")
        _cuda_dtype(probe, "probe", torch.complex64, "complex64")
        _cuda_dtype(positions_xy, "positions_xy", torch.long, "int64")
        sample, probe, pos = sample.contiguous(), probe.contiguous(), positions_xy.contiguous()
        dev = sample.device
        batch = pos.shape[0]
        ph, pw = probe.shape
        far = torch.empty((batch, ph, pw), dtype=torch.complex64, device=dev)
        amp = torch.empty((batch, ph, pw), dtype=torch.float32, device=dev)
        n = _abi.query("ptx_base_workspace_bytes", ph, pw, batch)
        ws = workspace(n, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_base_forward", ptr(sample), sample.shape[0], sample.shape[1], ptr(probe), ph, pw, ptr(pos),
                      batch, ptr(far), ptr(amp), ptr(ws), n, stream_handle(dev))
        patch_view = sample.as_strided((batch, ph, pw), (0, sample.shape[1], 1))
        return [patch_view, far, amp]

    @staticmethod
    def backward(grad_output, patch_stack, probe, far_field_shifted, positions_xy, sample_h: int, sample_w: int):
        _cuda_dtype(grad_output, "grad_output", torch.float32, "float32")
        _cuda_dtype(patch_stack, "patch_stack", torch.complex64, "complex64")
        _cuda_dtype(probe, "probe", torch.complex64, "complex64")
        _cuda_dtype(far_field_shifted, "far_field_shifted", torch.complex64, "complex64")
        _cuda_dtype(positions_xy, "positions_xy", torch.long, "int64")
        _check(patch_stack.dim() == 3 and patch_stack.stride(0) == 0 and patch_stack.stride(1) == sample_w,
               "patch_stack must be the sample view returned by this extension's forward")
        dev = probe.device
        batch = positions_xy.shape[0]
        ph, pw = probe.shape
        probe = probe.contiguous()
        grad_output = grad_output.contiguous()
        far = far_field_shifted.contiguous()
        pos = positions_xy.contiguous()
        gs = torch.empty((sample_h, sample_w), dtype=torch.complex64, device=dev)
        gp = torch.empty_like(probe)
        n = _abi.query("ptx_base_workspace_bytes", ph, pw, batch)
        ws = workspace(n, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_base_backward", ptr(grad_output), ptr(far), patch_stack.data_ptr(), sample_h, sample_w,
                      ptr(probe), ph, pw, ptr(pos), batch, ptr(gs), ptr(gp), ptr(ws), n, stream_handle(dev))
        return [gs, gp]

    @staticmethod
    def clear_plan_cache() -> None:
        _abi.call("ptx_clear_cache")


class _Fourier:
    """``ptychoX.fpm._C`` on libptychox (``fpm_extension.cpp:21-66``)."""

    @staticmethod
    def forward(object_field: torch.Tensor, pupil: torch.Tensor, led_indices_xy: torch.Tensor):
        _cuda_dtype(object_field, "object_field", torch.complex64, "complex64")
        _cuda_dtype(pupil, "pupil", torch.complex64, "complex64")
        _cuda_dtype(led_indices_xy, "led_indices_xy", torch.long, "int64")
        obj, pupil, led = object_field.contiguous(), pupil.contiguous(), led_indices_xy.contiguous()
        dev = obj.device
        batch = led.shape[0]
        (oh, ow), (lh, lw) = obj.shape, pupil.shape
        spectrum = torch.empty_like(obj)
        image = torch.empty((batch, lh, lw), dtype=torch.complex64, device=dev)
        amp = torch.empty((batch, lh, lw), dtype=torch.float32, device=dev)
        n = _abi.query("ptx_fpm_workspace_bytes", oh, ow, lh, lw, batch)
        ws = workspace(n, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_fpm_forward", ptr(obj), oh, ow, ptr(pupil), lh, lw, ptr(led), batch, ptr(spectrum),
                      ptr(image), ptr(amp), ptr(ws), n, stream_handle(dev))
        return [spectrum, image, amp]

    @staticmethod
    def backward(grad_output, sub_spectrum, pupil, image_field, led_indices_xy, object_h: int, object_w: int):
        _cuda_dtype(grad_output, "grad_output", torch.float32, "float32")
        _cuda_dtype(sub_spectrum, "sub_spectrum", torch.complex64, "complex64")
        _cuda_dtype(pupil, "pupil", torch.complex64, "complex64")
        _cuda_dtype(image_field, "image_field", torch.complex64, "complex64")
        _cuda_dtype(led_indices_xy, "led_indices_xy", torch.long, "int64")
        _check(tuple(sub_spectrum.shape) == (object_h, object_w),
               "sub_spectrum must be the object spectrum returned by this extension's forward")
        dev = pupil.device
        batch = led_indices_xy.shape[0]
        lh, lw = pupil.shape
        pupil, spectrum = pupil.contiguous(), sub_spectrum.contiguous()
        g, image, led = grad_output.contiguous(), image_field.contiguous(), led_indices_xy.contiguous()
        go = torch.empty((object_h, object_w), dtype=torch.complex64, device=dev)
        gp = torch.empty_like(pupil)
        n = _abi.query("ptx_fpm_workspace_bytes", object_h, object_w, lh, lw, batch)
        ws = workspace(n, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_fpm_backward", ptr(g), ptr(image), ptr(spectrum), object_h, object_w, ptr(pupil), lh, lw,
                      ptr(led), batch, ptr(go), ptr(gp), ptr(ws), n, stream_handle(dev))
        return [go, gp]

    @staticmethod
    def clear_plan_cache() -> None:
        _abi.call("ptx_clear_cache")


class _Coded:
    """``ptychoX.coded._C`` on libptychox (``coded_extension.cpp:26-94``)."""

    @staticmethod
    def forward(object_field, coded_surface, transfer_1, transfer_2, shifts_xy, downsample: int):
        for name, t in (("object", object_field), ("coded_surface", coded_surface), ("transfer_1", transfer_1),
                        ("transfer_2", transfer_2)):
            _cuda_dtype(t, name, torch.complex64, "complex64")
        _cuda_dtype(shifts_xy, "shifts_xy", torch.float32, "float32")
        obj, mask = object_field.contiguous(), coded_surface.contiguous()
        t1, t2, shifts = transfer_1.contiguous(), transfer_2.contiguous(), shifts_xy.contiguous()
        dev = obj.device
        n = obj.shape[0]
        batch = shifts.shape[0]
        ds = int(downsample)
        xf = torch.empty((batch, n, n), dtype=torch.complex64, device=dev)
        sensor = torch.empty_like(xf)
        amp = torch.empty((batch, n // ds, n // ds), dtype=torch.float32, device=dev)
        nb = _abi.query("ptx_coded_workspace_bytes", n, batch)
        ws = workspace(nb, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_coded_forward", ptr(obj), ptr(mask), ptr(t1), ptr(t2), n, ptr(shifts), batch, ds, ptr(xf),
                      ptr(sensor), ptr(amp), ptr(ws), nb, stream_handle(dev))
        return [amp.clone(), xf, sensor, amp]

    @staticmethod
    def backward(grad_output, object_spectrum, x_forward, sensor_field, coded_surface, transfer_1, transfer_2,
                 shifts_xy, downsample: int):
        _cuda_dtype(grad_output, "grad_output", torch.float32, "float32")
        _cuda_dtype(object_spectrum, "object_spectrum", torch.float32, "the pooled amplitude returned by forward")
        for name, t in (("x_forward", x_forward), ("sensor_field", sensor_field), ("coded_surface", coded_surface),
                        ("transfer_1", transfer_1), ("transfer_2", transfer_2)):
            _cuda_dtype(t, name, torch.complex64, "complex64")
        dev = x_forward.device
        batch, n = x_forward.shape[0], x_forward.shape[1]
        ds = int(downsample)
        g, amp = grad_output.contiguous(), object_spectrum.contiguous()
        xf, sensor, mask = x_forward.contiguous(), sensor_field.contiguous(), coded_surface.contiguous()
        t1, t2, shifts = transfer_1.contiguous(), transfer_2.contiguous(), shifts_xy.contiguous()
        go = torch.empty((n, n), dtype=torch.complex64, device=dev)
        gm = torch.empty_like(go)
        nb = _abi.query("ptx_coded_workspace_bytes", n, batch)
        ws = workspace(nb, dev)
        with torch.cuda.device(dev):
            _abi.call("ptx_coded_backward", ptr(g), ptr(xf), ptr(sensor), ptr(amp), ptr(mask), ptr(t1), ptr(t2), n,
                      ptr(shifts), batch, ds, ptr(go), ptr(gm), ptr(ws), nb, stream_handle(dev))
        return [go, gm]

    @staticmethod
    def clear_plan_cache() -> None:
        _abi.call("ptx_clear_cache")


BASE = _Base()
FOURIER = _Fourier()
CODED = _Coded()


def install(ptychoX_package) -> None:
    """Route an imported reference package's CUDA path to libptychox.

    Sets the module-level ``_CUDA_EXT`` of ``ptychoX.base.ops``, ``ptychoX.fpm.ops`` and
    ``ptychoX.coded.ops``, which each ``_load_cuda_ext`` returns once set; the reference's
    operators then call these objects whenever ``use_cuda_kernels=True`` and the tensors are
    CUDA complex64 (``_utils.can_use_cuda_ext``)."""
    import importlib

    _abi.load()
    name = ptychoX_package.__name__
    for sub, ext in (("base", BASE), ("fpm", FOURIER), ("coded", CODED)):
        mod = importlib.import_module(f"{name}.{sub}.ops")
        mod._CUDA_EXT = ext
