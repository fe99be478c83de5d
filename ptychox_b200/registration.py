"""Sub-pixel image registration for positional tracking of coded / near-field scans.

Mirrors the MATLAB helpers of the reference's near-field example
(``matlab/Examples/Near-field Ptychography/+misc``):

* ``dftregistration`` — ``dftregistration.m:70-138``: efficient sub-pixel registration by
  cross-correlation (M. Guizar-Sicairos, S. T. Thurman and J. R. Fienup, Opt. Lett. 33,
  156-158 (2008)), batched over images;
* ``track_position`` — ``track_position.m:24-41`` (register every measurement against
  the first, 20-pixel border removed, ``usfac = 600``);
* ``refine_position`` — ``refine_position.m:25-55`` (register against the average of the
  measurements shifted back by their initial estimates, ``usfac = 100``).

Stacks are ``[n, h, w]`` (the MATLAB functions take ``[h, w, n]``); shifts are
``(row, col)`` as in the reference, and the trackers return ``(locX, locY)`` =
``(col, row)``.  The plain FFTs of images and the 2x zero-padded cross-correlation run on
cuFFT (``torch.fft``); the matrix-multiply DFT refinement (``dftups``, ``:150-185``) and
its peak search run in libptychox (``ptx_reg_upsampled_peak``, summed in FP64).  FP32
spectra and FFTs, FP64 energy sums.
"""

from __future__ import annotations

import math

import torch

from . import _abi
from ._utils import ptr, stream_handle, workspace

__all__ = ["dftregistration", "track_position", "refine_position"]

_WS_CAP = 2 << 30  # refinement workspace per library call; larger batches are split


def _freq(n: int, device) -> torch.Tensor:
    """``ifftshift(-fix(n/2):ceil(n/2)-1)`` (``dftregistration.m:73-74``)."""
    return torch.fft.ifftshift(torch.arange(-(n // 2), (n + 1) // 2, device=device))


def _argmax_colmajor(a: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """(row, col) of the first maximum of each ``[B, R, C]`` slice in column-major order
    (MATLAB's ``find(A == max(A(:)), 1, 'first')``)."""
    rows = a.shape[1]
    idx = a.transpose(1, 2).reshape(a.shape[0], -1).argmax(dim=1)
    return idx % rows, idx // rows


def _round_matlab(x: torch.Tensor) -> torch.Tensor:
    return torch.sign(x) * torch.floor(x.abs() + 0.5)


def _ftpad2(spec: torch.Tensor) -> torch.Tensor:
    """``FTpad(spec, [2 nr, 2 nc])`` (``dftregistration.m:189-224``) for ``[B, nr, nc]``."""
    b, nr, nc = spec.shape
    out = torch.zeros(b, 2 * nr, 2 * nc, dtype=spec.dtype, device=spec.device)
    r0, c0 = nr - nr // 2, nc - nc // 2
    out[:, r0:r0 + nr, c0:c0 + nc] = torch.fft.fftshift(spec, dim=(-2, -1))
    return torch.fft.ifftshift(out, dim=(-2, -1)) * 4.0


def _refine(q: torch.Tensor, usfac: int, rc: torch.Tensor, cc: torch.Tensor):
    """Peak (row, col) of the upsampled patch and CC there, through the library."""
    b, nr, nc = q.shape
    peak_rc = torch.empty(b, 2, dtype=torch.int32, device=q.device)
    peak_cc = torch.empty(b, dtype=torch.complex128, device=q.device)
    per_image = max(1, _abi.query("ptx_reg_workspace_bytes", 1, nr, nc, usfac))
    step = max(1, min(b, _WS_CAP // per_image))
    ws = workspace(per_image * step, q.device)
    with torch.cuda.device(q.device):
        for s in range(0, b, step):
            e = min(b, s + step)
            _abi.call("ptx_reg_upsampled_peak", ptr(q[s:e]), e - s, nr, nc, int(usfac), ptr(rc[s:e]), ptr(cc[s:e]),
                      ptr(peak_rc[s:e]), ptr(peak_cc[s:e]), ptr(ws), ws.numel(), stream_handle(q.device))
    return peak_rc.long(), peak_cc


def dftregistration(buf1ft: torch.Tensor, buf2ft: torch.Tensor, usfac: int = 1, return_registered: bool = False):
    """``[error, diffphase, row_shift, col_shift]`` registering ``buf2ft`` to ``buf1ft``.

    ``buf1ft`` / ``buf2ft``: complex spectra (``fft2`` of the images) on the GPU, ``[h, w]``
    or ``[B, h, w]`` (a single spectrum on either side is broadcast).  ``usfac``: 0 (error
    and phase only), 1 (whole pixels), 2 (half pixels) or larger (1/usfac of a pixel).
    Returns float64 ``[B, 4]``, or ``[4]`` when both inputs are 2-D; with
    ``return_registered`` also ``Greg``, the spectrum of ``buf2ft`` shifted and phase-corrected
    onto ``buf1ft`` (the second output of ``dftregistration.m:140-148``), complex64.
    """
    if buf1ft.ndim not in (2, 3) or buf2ft.ndim not in (2, 3):
        raise ValueError("buf1ft and buf2ft must be [h, w] or [batch, h, w] spectra.")
    if not buf1ft.is_cuda or not buf2ft.is_cuda:
        raise ValueError("buf1ft and buf2ft must be CUDA tensors (ptychox_b200 has no CPU path).")
    if buf1ft.shape[-2:] != buf2ft.shape[-2:]:
        raise ValueError("buf1ft and buf2ft must have the same image size.")
    usfac = int(usfac)
    if usfac < 0:
        raise ValueError("usfac must be non-negative.")
    single = buf1ft.ndim == 2 and buf2ft.ndim == 2
    b1 = buf1ft.to(torch.complex64).reshape(-1, *buf1ft.shape[-2:])
    b2 = buf2ft.to(torch.complex64).reshape(-1, *buf2ft.shape[-2:])
    bsz = max(b1.shape[0], b2.shape[0])
    b1, b2 = b1.expand(bsz, -1, -1), b2.expand(bsz, -1, -1)
    nr, nc = b2.shape[-2:]
    dev = b2.device
    ar = torch.arange(bsz, device=dev)
    zeros = torch.zeros(bsz, dtype=torch.float64, device=dev)
    if usfac == 0:
        ccmax = (b1.to(torch.complex128) * b2.to(torch.complex128).conj()).sum(dim=(-2, -1))
        row_shift, col_shift = zeros, zeros.clone()
    elif usfac == 1:
        cc = torch.fft.ifft2(b1 * b2.conj())
        r, c = _argmax_colmajor(cc.abs())
        ccmax = cc[ar, r, c].to(torch.complex128) * (nr * nc)
        row_shift, col_shift = _freq(nr, dev)[r].double(), _freq(nc, dev)[c].double()
    else:
        cc = torch.fft.ifft2(_ftpad2(b1 * b2.conj()))
        r, c = _argmax_colmajor(cc.abs())
        ccmax = cc[ar, r, c].to(torch.complex128) * (nr * nc)
        row_shift = torch.fft.ifftshift(torch.arange(-nr, nr, device=dev))[r].double() / 2.0
        col_shift = torch.fft.ifftshift(torch.arange(-nc, nc, device=dev))[c].double() / 2.0
        if usfac > 2:
            rc = _round_matlab(row_shift * usfac)
            ccn = _round_matlab(col_shift * usfac)
            q = (b2 * b1.conj()).contiguous()
            peak, ccmax = _refine(q, usfac, rc.to(torch.int32).contiguous(), ccn.to(torch.int32).contiguous())
            dftshift = math.ceil(1.5 * usfac) // 2
            ccmax = ccmax.to(torch.complex128)
            row_shift = rc / usfac + (peak[:, 0] - dftshift).double() / usfac
            col_shift = ccn / usfac + (peak[:, 1] - dftshift).double() / usfac
        if nr == 1:
            row_shift = zeros
        if nc == 1:
            col_shift = zeros.clone()
    rg00 = (b1.abs().double() ** 2).sum(dim=(-2, -1))
    rf00 = (b2.abs().double() ** 2).sum(dim=(-2, -1))
    error = torch.sqrt(torch.abs(1.0 - ccmax.abs() ** 2 / (rg00 * rf00)))
    diffphase = torch.angle(ccmax)
    out = torch.stack([error, diffphase, row_shift, col_shift], dim=1)
    if not return_registered:
        return out[0] if single else out
    fr = _freq(nr, dev).double()[None, :, None] / nr
    fc = _freq(nc, dev).double()[None, None, :] / nc
    phase = diffphase[:, None, None]
    if usfac > 0:
        phase = phase - 2 * math.pi * (row_shift[:, None, None] * fr + col_shift[:, None, None] * fc)
    greg = b2 * torch.polar(torch.ones_like(phase), phase).to(torch.complex64)
    return (out[0], greg[0]) if single else (out, greg)


def _crop(stack: torch.Tensor, edge: int) -> torch.Tensor:
    return stack[..., edge:stack.shape[-2] - edge, edge:stack.shape[-1] - edge]


def _check_stack(im_raw_crop: torch.Tensor, edge: int) -> torch.Tensor:
    if im_raw_crop.ndim != 3:
        raise ValueError("im_raw_crop must be an [n, h, w] stack.")
    if not im_raw_crop.is_cuda:
        raise ValueError("im_raw_crop must be a CUDA tensor (ptychox_b200 has no CPU path).")
    if min(im_raw_crop.shape[-2:]) <= 2 * edge:
        raise ValueError(f"images must be larger than twice the {edge}-pixel border.")
    return im_raw_crop.to(torch.float32)


def track_position(im_raw_crop: torch.Tensor, edge: int = 20, usfac: int = 600, return_registered: bool = False):
    """Initial positional tracking (``track_position.m:24-41``): every measurement of the
    ``[n, h, w]`` stack registered against the first, ``edge`` pixels of border removed.
    Returns float64 ``(locX, locY)``, and with ``return_registered`` also ``regi``, the
    registered spectra of the cropped measurements (``[n, h - 2 edge, w - 2 edge]``)."""
    stack = _check_stack(im_raw_crop, edge)
    spectra = torch.fft.fft2(_crop(stack, edge).to(torch.complex64))
    res = dftregistration(spectra[0], spectra, usfac, return_registered=return_registered)
    if return_registered:
        out, regi = res
        return out[:, 3], out[:, 2], regi
    return res[:, 3], res[:, 2]


def refine_position(im_raw_crop: torch.Tensor, loc_x0, loc_y0, edge: int = 20, usfac: int = 100):
    """Positional refinement (``refine_position.m:25-55``): the stack is normalised by its
    mean image; the measurements whose initial shifts both exceed 2 pixels in magnitude are
    shifted back by them (Fourier phase ramp) and averaged (magnitude) into a reference, and
    every measurement is registered against it.  Returns float64 ``(locX, locY)``."""
    stack = _check_stack(im_raw_crop, edge)
    stack = stack / stack.mean(dim=0, keepdim=True)
    n, h, w = stack.shape
    dev = stack.device
    x0 = torch.as_tensor(loc_x0, dtype=torch.float64, device=dev).reshape(n)
    y0 = torch.as_tensor(loc_y0, dtype=torch.float64, device=dev).reshape(n)
    fy = _freq(h, dev).double()[:, None]
    fx = _freq(w, dev).double()[None, :]
    use = torch.nonzero((x0.abs() > 2) & (y0.abs() > 2)).flatten()
    ref = torch.zeros(h, w, dtype=torch.complex64, device=dev)
    for s in range(0, use.numel(), 64):
        idx = use[s:s + 64]
        hs = torch.exp(-2j * math.pi * (fx * x0[idx, None, None] / w + fy * y0[idx, None, None] / h))
        ref += torch.fft.ifft2(torch.fft.fft2(stack[idx].to(torch.complex64)) * hs.to(torch.complex64)).sum(dim=0)
    ref_img = ref.abs() / n
    ref_ft = torch.fft.fft2(_crop(ref_img, edge).to(torch.complex64))
    out = dftregistration(ref_ft, torch.fft.fft2(_crop(stack, edge).to(torch.complex64)), usfac)
    return out[:, 3], out[:, 2]
