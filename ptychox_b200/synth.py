"""Seeded synthetic inputs for the four modalities (host side, numpy; the measurement
synthesis also on the device).

The reference drivers build their problems from images on disk (``cameraman512.png``,
``I01.bmp``); the workloads here use seeded synthetic objects of the same shapes:

* objects: amplitude ``U[0.8, 1]``, phase ``U[-pi/2, pi/2]`` per pixel;
* conventional probe: Gaussian apodisation times a smooth random phase screen (a
  diffuser), so far fields are speckle and no detector pixel saturates uint16;
* raster scans with integer jitter (``train_ptychography.py:377-397`` draws random
  positions; the configs specify a raster plus ``U[-j, j]`` jitter);
* FPM: circular pupil and LED-grid windows (``train_fpm.py:38-52,105-120`` geometry);
* coded / near-field: angular-spectrum transfer functions exactly as
  ``train_coded.py:50-65``, a binary random mask at 50% fill, and sub-pixel shifts
  normalised by the field side (``train_coded.py:68-70,159``);
* measurements: Poisson counts of ``|model|^2 / scale`` stored as uint16, with one
  global ``scale`` chosen so an average pattern holds the requested photon count; on the
  device, ``synthesize_dataset`` (the reference's chunked forward,
  ``train_ptychography.py:432-450``) and ``poisson_counts_device`` draw them without a
  host round trip.
"""

from __future__ import annotations

import math

import numpy as np

__all__ = [
    "random_object",
    "gaussian_probe",
    "raster_positions",
    "poisson_counts",
    "circular_pupil",
    "fpm_led_windows",
    "fpm_dx_for_pupil",
    "angular_spectrum_transfer",
    "binary_mask",
    "coded_shifts",
    "synthesize_dataset",
    "poisson_counts_device",
]


def random_object(h: int, w: int | None = None, rng: np.random.Generator | None = None) -> np.ndarray:
    """complex64 ``[h, w]``: amplitude ``U[0.8, 1]``, phase ``U[-pi/2, pi/2]``."""
    rng = rng or np.random.default_rng(0)
    w = h if w is None else w
    amp = rng.uniform(0.8, 1.0, size=(h, w))
    phase = rng.uniform(-math.pi / 2, math.pi / 2, size=(h, w))
    return (amp * np.exp(1j * phase)).astype(np.complex64)


def _smooth_noise(h: int, w: int, corr: float, rng: np.random.Generator) -> np.ndarray:
    noise = rng.standard_normal((h, w))
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.fftfreq(w)[None, :]
    filt = np.exp(-(fx**2 + fy**2) * (corr**2) * 2.0 * math.pi**2)
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    return field / (field.std() + 1e-12)


def gaussian_probe(h: int, w: int | None = None, rng: np.random.Generator | None = None,
                   sigma_frac: float = 0.2, phase_rad: float = 2.0, corr_frac: float = 0.03) -> np.ndarray:
    """complex64 Gaussian-apodised probe with a smooth random phase screen."""
    rng = rng or np.random.default_rng(0)
    w = h if w is None else w
    yy = (np.arange(h) - (h - 1) / 2.0)[:, None]
    xx = (np.arange(w) - (w - 1) / 2.0)[None, :]
    sig_y, sig_x = sigma_frac * h, sigma_frac * w
    amp = np.exp(-0.5 * ((yy / sig_y) ** 2 + (xx / sig_x) ** 2))
    phase = phase_rad * _smooth_noise(h, w, corr_frac * max(h, w), rng)
    return (amp * np.exp(1j * phase)).astype(np.complex64)


def raster_positions(grid: int, step: int, origin: int, jitter: int,
                     rng: np.random.Generator | None = None, grid_x: int | None = None) -> np.ndarray:
    """int64 ``[grid*grid_x, 2]`` zero-based ``(x, y)`` raster with integer ``U[-j, j]`` jitter."""
    rng = rng or np.random.default_rng(0)
    gx = grid if grid_x is None else grid_x
    ys, xs = np.meshgrid(np.arange(grid), np.arange(gx), indexing="ij")
    pos = np.stack([origin + xs.ravel() * step, origin + ys.ravel() * step], axis=1).astype(np.int64)
    if jitter:
        pos = pos + rng.integers(-jitter, jitter + 1, size=pos.shape)
    return pos


def raster_positions_subpixel(grid: int, step: int, origin: int, jitter: float,
                              rng: np.random.Generator | None = None, grid_x: int | None = None) -> np.ndarray:
    """float64 ``[grid*grid_x, 2]`` zero-based ``(x, y)`` raster with real ``U[-j, j]`` jitter
    (sub-pixel scan positions)."""
    rng = rng or np.random.default_rng(0)
    gx = grid if grid_x is None else grid_x
    ys, xs = np.meshgrid(np.arange(grid), np.arange(gx), indexing="ij")
    pos = np.stack([origin + xs.ravel() * step, origin + ys.ravel() * step], axis=1).astype(np.float64)
    if jitter:
        pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    return pos


def poisson_counts(model_intensity: np.ndarray, photons: float, rng: np.random.Generator | None = None,
                   per_pixel: bool = False, brightest: bool = False) -> tuple[np.ndarray, float]:
    """Poisson uint16 counts of ``I / scale`` and the ``scale`` that decodes them.

    ``scale`` makes an average pattern (or, with ``brightest``, the brightest pattern) hold
    ``photons`` counts in total — with ``per_pixel``, ``photons`` counts per pixel on
    average.  The decoded amplitude is ``sqrt(scale * counts)``.  Raises if any count
    exceeds uint16.
    """
    rng = rng or np.random.default_rng(0)
    inten = np.asarray(model_intensity, dtype=np.float64)
    sums = inten.reshape(inten.shape[0], -1).sum(axis=1)
    per_pattern = sums.max() if brightest else sums.mean()
    denom = photons if not per_pixel else photons * inten[0].size
    scale = float(per_pattern / denom)
    counts = rng.poisson(inten / scale)
    if counts.max() > 65535:
        raise ValueError(f"Poisson counts saturate uint16 (max {counts.max()}); lower the photon count")
    return counts.astype(np.uint16), float(np.float32(scale))


def circular_pupil(h: int, radius_frac: float) -> np.ndarray:
    """complex64 ``[h, h]`` circular aperture of radius ``radius_frac * h`` around the centre.

    The pupil is indexed like the window it multiplies (fftshifted spectrum, DC at
    ``h // 2``), as in ``fpm/ops.py:181-182``.
    """
    c = h // 2
    yy, xx = np.meshgrid(np.arange(h) - c, np.arange(h) - c, indexing="ij")
    return ((yy**2 + xx**2) <= (radius_frac * h) ** 2).astype(np.complex64)


def fpm_led_windows(n_high: int, n_low: int, grid: int, pitch_mm: float, height_mm: float,
                    wavelength_um: float, dx_high_um: float) -> np.ndarray:
    """int64 ``[grid*grid, 2]`` ``(x, y)`` window corners in the fftshifted high-res spectrum.

    LED ``(i, j)`` at ``((i - c) pitch, (j - c) pitch, height)`` illuminates with spatial
    frequency ``sin(theta) / lambda``; in spectrum pixels that is
    ``round(sin(theta) / lambda * n_high * dx)``, and the window corner is that shift plus
    the centred corner ``(n_high - n_low) // 2``.  Raises if a window leaves the spectrum.
    """
    c = (grid - 1) / 2.0
    out = []
    base = (n_high - n_low) // 2
    for j in range(grid):
        for i in range(grid):
            x = (i - c) * pitch_mm
            y = (j - c) * pitch_mm
            r = math.sqrt(x * x + y * y + height_mm * height_mm)
            kx = x / r / wavelength_um * n_high * dx_high_um
            ky = y / r / wavelength_um * n_high * dx_high_um
            out.append((base + int(round(kx)), base + int(round(ky))))
    led = np.asarray(out, dtype=np.int64)
    if led.min() < 0 or led.max() > n_high - n_low:
        raise ValueError("an LED window leaves the high-resolution spectrum")
    return led


def fpm_dx_for_pupil(n_high: int, n_low: int, na: float, wavelength_um: float, radius_frac: float) -> float:
    """High-res pixel size (um) that puts the pupil edge ``NA / lambda`` at ``radius_frac * n_low``.

    A spectrum pixel of the ``n_high`` grid is ``1 / (n_high dx)``, so the pupil radius in
    pixels is ``NA / lambda * n_high * dx``.
    """
    return radius_frac * n_low * wavelength_um / (na * n_high)


def angular_spectrum_transfer(n: int, pixel_size: float, wavelength: float, distance: float) -> np.ndarray:
    """complex64 angular-spectrum transfer function (``train_coded.py:50-65``), unshifted."""
    freq = np.fft.fftfreq(n, d=pixel_size)
    fy, fx = np.meshgrid(freq, freq, indexing="ij")
    inv_lambda = 1.0 / wavelength
    kz_sq = inv_lambda**2 - fx**2 - fy**2
    kz_real = np.sqrt(np.clip(kz_sq, 0.0, None))
    evanescent = np.sqrt(np.clip(-kz_sq, 0.0, None))
    phase = np.exp(1j * 2.0 * math.pi * distance * kz_real)
    decay = np.exp(-2.0 * math.pi * abs(distance) * evanescent)
    return (phase * decay * (kz_sq >= 0)).astype(np.complex64)


def binary_mask(n: int, fill: float = 0.5, rng: np.random.Generator | None = None) -> np.ndarray:
    """complex64 binary random coded surface at the given fill factor."""
    rng = rng or np.random.default_rng(0)
    return (rng.random((n, n)) < fill).astype(np.complex64)


def coded_shifts(count: int, max_px: float, n: int, rng: np.random.Generator | None = None) -> np.ndarray:
    """float32 ``[count, 2]`` shifts ``U[-max_px, max_px] / n`` (field-normalised)."""
    rng = rng or np.random.default_rng(0)
    px = rng.uniform(-max_px, max_px, size=(count, 2))
    return (px / n).astype(np.float32)


def synthesize_dataset(object_true, probe_true, positions, batch_size: int):
    """Forward amplitudes of every scan position, ``batch_size`` positions per operator call.

    The reference's ``synthesize_dataset`` (``train_ptychography.py:432-450``, under
    ``torch.no_grad``): ``ptychoX_base`` over consecutive slices of ``positions``,
    concatenated along the batch.  Tensors as for ``ptychoX_base``.
    """
    import torch

    from .base import ptychoX_base

    if batch_size <= 0:
        raise ValueError("batch_size must be positive.")
    with torch.no_grad():
        chunks = [ptychoX_base(object_true, probe_true, positions[s:s + batch_size])
                  for s in range(0, positions.shape[0], batch_size)]
    return torch.cat(chunks, dim=0)


def poisson_counts_device(amplitude, photons: float, seed: int = 0, per_pixel: bool = False,
                          brightest: bool = False):
    """Device twin of ``poisson_counts`` for amplitudes already on the GPU.

    Returns uint16 Poisson counts of ``amplitude**2 / scale`` drawn with torch's device RNG
    (seeded with ``seed``) and ``scale`` (a float32 value, used for the draw as well), with
    ``scale`` chosen as in ``poisson_counts``.  Raises if any count exceeds uint16.
    """
    import torch

    inten = amplitude.double() ** 2
    sums = inten.flatten(1).sum(dim=1)
    per_pattern = float(sums.max() if brightest else sums.mean())
    denom = photons * (inten[0].numel() if per_pixel else 1)
    scale = float(np.float32(per_pattern / denom))
    gen = torch.Generator(device=amplitude.device).manual_seed(seed)
    counts = torch.poisson(inten / scale, generator=gen)
    if float(counts.max()) > 65535:
        raise ValueError("Poisson counts saturate uint16; lower the photon count")
    return counts.to(torch.int32).to(torch.uint16), scale
