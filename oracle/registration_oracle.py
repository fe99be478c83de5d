"""CPU oracle for sub-pixel image registration (positional tracking of coded / near-field scans).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker of
``ptychox_b200.registration``; the product never imports it.

It restates, in numpy (FP64), the MATLAB helpers of the reference's near-field example
(``matlab/Examples/Near-field Ptychography/+misc``):

* ``dftregistration.m:1-148``: efficient sub-pixel registration by cross-correlation
  (M. Guizar-Sicairos, S. T. Thurman and J. R. Fienup, "Efficient subpixel image
  registration algorithms", Opt. Lett. 33, 156-158 (2008)): a 2x zero-padded FFT
  cross-correlation for the initial peak (``:90-101``), then a matrix-multiply DFT
  upsampled by ``usfac`` in a 1.5-pixel neighbourhood of it (``:102-121``), error and
  phase difference from the peak value (``:132-138``);
* ``dftups`` (``:150-185``) and ``FTpad`` (``:189-224``), its two helpers, and the
  registered spectrum ``Greg`` (``:140-148``);
* ``track_position.m:24-41`` and ``refine_position.m:25-55``: register every cropped
  measurement against a reference image (the first measurement, or the average of the
  measurements shifted back by their initial estimates) with a 20-pixel border removed.

MATLAB's ``find(A == max(A(:)), 1, 'first')`` returns the first maximum in column-major
order; ``_argmax_colmajor`` keeps that tie rule.  Shifts are ``(row, col)`` as in the
reference (``locY = row``, ``locX = col``).

Parity pin: there is no runnable MATLAB here, so the restatement is checked against the
algorithm's defining property instead (``tests/test_registration_oracle.py``): images
shifted by known sub-pixel amounts through a Fourier phase ramp are registered to
within half a grid step of 1/usfac, and the usfac = 2 and usfac = 1 branches agree with
a brute-force DFT cross-correlation.
"""

from __future__ import annotations

import numpy as np

__all__ = ["dftregistration", "registered", "dftups", "ftpad", "track_position", "refine_position"]


def _fix(x: float) -> int:
    return int(np.trunc(x))


def _freq(n: int) -> np.ndarray:
    """``ifftshift(-fix(n/2):ceil(n/2)-1)`` (``dftregistration.m:73-74``)."""
    return np.fft.ifftshift(np.arange(-_fix(n / 2), int(np.ceil(n / 2))))


def _round_matlab(x: float) -> float:
    """MATLAB ``round``: halves away from zero."""
    return float(np.sign(x) * np.floor(abs(x) + 0.5))


def _argmax_colmajor(a: np.ndarray) -> tuple[int, int]:
    """Zero-based (row, col) of the first maximum in column-major order."""
    flat = np.argmax(a.T.ravel())  # numpy returns the first maximum of the flattened order
    c, r = divmod(int(flat), a.shape[0])
    return r, c


def ftpad(im_ft: np.ndarray, outsize: tuple[int, int]) -> np.ndarray:
    """Zero-pad (or crop) a spectrum around its centre, scaled to keep the mean
    (``dftregistration.m:189-224``)."""
    nin = np.array(im_ft.shape)
    nout = np.array(outsize)
    f = np.fft.fftshift(im_ft)
    center = nin // 2 + 1
    centerout = nout // 2 + 1
    cc = centerout - center
    out = np.zeros(outsize, dtype=np.complex128)
    r0o, r1o = max(cc[0] + 1, 1), min(cc[0] + nin[0], nout[0])
    c0o, c1o = max(cc[1] + 1, 1), min(cc[1] + nin[1], nout[1])
    r0i, r1i = max(-cc[0] + 1, 1), min(-cc[0] + nout[0], nin[0])
    c0i, c1i = max(-cc[1] + 1, 1), min(-cc[1] + nout[1], nin[1])
    out[r0o - 1:r1o, c0o - 1:c1o] = f[r0i - 1:r1i, c0i - 1:c1i]
    return np.fft.ifftshift(out) * (nout[0] * nout[1]) / (nin[0] * nin[1])


def dftups(x: np.ndarray, nor: int, noc: int, usfac: int, roff: float, coff: float) -> np.ndarray:
    """Upsampled DFT by matrix multiplies (``dftregistration.m:150-185``): ``nor x noc``
    samples of the inverse DFT of ``x``, upsampled by ``usfac``, the output origin at
    ``(roff, coff)`` of the upsampled grid."""
    nr, nc = x.shape
    fc = np.fft.ifftshift(np.arange(nc)) - nc // 2
    fr = np.fft.ifftshift(np.arange(nr)) - nr // 2
    kernc = np.exp((-2j * np.pi / (nc * usfac)) * np.outer(fc, np.arange(noc) - coff))
    kernr = np.exp((-2j * np.pi / (nr * usfac)) * np.outer(np.arange(nor) - roff, fr))
    return kernr @ x @ kernc


def registered(buf2ft: np.ndarray, output: np.ndarray, usfac: int) -> np.ndarray:
    """``Greg`` (``dftregistration.m:140-148``): ``buf2ft`` shifted by the registration
    output and multiplied by ``exp(i diffphase)``."""
    nr, nc = buf2ft.shape
    ncg, nrg = np.meshgrid(_freq(nc), _freq(nr))
    g = np.asarray(buf2ft, dtype=np.complex128)
    if usfac > 0:
        g = g * np.exp(2j * np.pi * (-output[2] * nrg / nr - output[3] * ncg / nc))
    return g * np.exp(1j * output[1])


def dftregistration(buf1ft: np.ndarray, buf2ft: np.ndarray, usfac: int = 1) -> np.ndarray:
    """``[error, diffphase, row_shift, col_shift]`` registering ``buf2ft`` to ``buf1ft``
    (both spectra, ``fft2`` of the images; ``dftregistration.m:70-138``)."""
    buf1ft = np.asarray(buf1ft, dtype=np.complex128)
    buf2ft = np.asarray(buf2ft, dtype=np.complex128)
    nr, nc = buf2ft.shape
    nr1, nc1 = _freq(nr), _freq(nc)
    if usfac == 0:
        ccmax = np.sum(buf1ft * np.conj(buf2ft))
        row_shift = col_shift = 0.0
    elif usfac == 1:
        cc = np.fft.ifft2(buf1ft * np.conj(buf2ft))
        r, c = _argmax_colmajor(np.abs(cc))
        ccmax = cc[r, c] * nr * nc
        row_shift, col_shift = float(nr1[r]), float(nc1[c])
    else:
        cc = np.fft.ifft2(ftpad(buf1ft * np.conj(buf2ft), (2 * nr, 2 * nc)))
        r, c = _argmax_colmajor(np.abs(cc))
        ccmax = cc[r, c] * nr * nc
        nr2 = np.fft.ifftshift(np.arange(-nr, nr))
        nc2 = np.fft.ifftshift(np.arange(-nc, nc))
        row_shift, col_shift = nr2[r] / 2.0, nc2[c] / 2.0
        if usfac > 2:
            row_shift = _round_matlab(row_shift * usfac) / usfac
            col_shift = _round_matlab(col_shift * usfac) / usfac
            n_out = int(np.ceil(usfac * 1.5))
            dftshift = _fix(n_out / 2)
            cc = np.conj(dftups(buf2ft * np.conj(buf1ft), n_out, n_out, usfac,
                                dftshift - row_shift * usfac, dftshift - col_shift * usfac))
            r, c = _argmax_colmajor(np.abs(cc))
            ccmax = cc[r, c]
            row_shift = row_shift + (r - dftshift) / usfac
            col_shift = col_shift + (c - dftshift) / usfac
        if nr == 1:
            row_shift = 0.0
        if nc == 1:
            col_shift = 0.0
    rg00 = np.sum(np.abs(buf1ft) ** 2)
    rf00 = np.sum(np.abs(buf2ft) ** 2)
    error = np.sqrt(np.abs(1.0 - np.abs(ccmax) ** 2 / (rg00 * rf00)))
    return np.array([error, np.angle(ccmax), row_shift, col_shift])


def _crop(stack: np.ndarray, edge: int) -> np.ndarray:
    return stack[..., edge:stack.shape[-2] - edge, edge:stack.shape[-1] - edge]


def track_position(im_raw_crop: np.ndarray, edge: int = 20, usfac: int = 600) -> tuple[np.ndarray, np.ndarray]:
    """Initial tracking (``track_position.m:24-41``): register every measurement of the
    ``[n, h, w]`` stack against the first, border removed.  Returns ``(locX, locY)``."""
    stack = np.asarray(im_raw_crop, dtype=np.float64)
    ref = np.fft.fft2(_crop(stack[0], edge))
    out = np.array([dftregistration(ref, np.fft.fft2(_crop(im, edge)), usfac) for im in stack])
    return out[:, 3], out[:, 2]


def refine_position(im_raw_crop: np.ndarray, loc_x0, loc_y0, edge: int = 20,
                    usfac: int = 100) -> tuple[np.ndarray, np.ndarray]:
    """Refinement (``refine_position.m:25-55``): normalise by the mean image, average the
    measurements shifted back by their initial estimates (those with both ``|shift| > 2``)
    into a reference, register every measurement against it.  Returns ``(locX, locY)``."""
    stack = np.asarray(im_raw_crop, dtype=np.float64)
    stack = stack / stack.mean(axis=0, keepdims=True)
    n, h, w = stack.shape
    fy = np.fft.ifftshift(np.arange(-(h // 2), int(np.ceil(h / 2))))
    fx = np.fft.ifftshift(np.arange(-(w // 2), int(np.ceil(w / 2))))
    fxx, fyy = np.meshgrid(fx, fy)
    acc = np.zeros((h, w), dtype=np.complex128)
    for i in range(n):
        x0, y0 = float(loc_x0[i]), float(loc_y0[i])
        if abs(x0) > 2 and abs(y0) > 2:
            hs = np.exp(-2j * np.pi * (fxx * x0 / w + fyy * y0 / h))
            acc += np.fft.ifft2(np.fft.fft2(stack[i]) * hs)
    ref = np.fft.fft2(_crop(np.abs(acc) / n, edge))
    out = np.array([dftregistration(ref, np.fft.fft2(_crop(im, edge)), usfac) for im in stack])
    return out[:, 3], out[:, 2]
