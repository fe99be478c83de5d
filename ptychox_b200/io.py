"""Reconstruction files in the reference drivers' format.

The reference's training scripts end by writing one ``torch.save`` dictionary per run:

* conventional, ``reconstruction.pt`` (``train_ptychography.py:588-597``): ``sample``,
  ``probe``, ``positions_xy``, ``observed_amplitude``, ``args``;
* Fourier, ``fpm_reconstruction.pt`` (``train_fpm.py:303-312``): ``object``, ``pupil``,
  ``led_indices_xy``, ``observed_amplitude``, ``args``;
* coded / near-field, ``coded_reconstruction.pt`` (``train_coded.py:284-293``): ``object``,
  ``coded_surface``, ``shifts_xy_pixels``, ``observed_amplitude``, ``args``.

``save_reconstruction`` writes the same dictionaries (CPU tensors, so the reference's tools
read them unchanged) from this library's results; ``load_reconstruction`` reads a file of
either origin back.  The per-epoch PNG previews the reference writes next to them belong to
its viewers and are not produced here.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

__all__ = ["FILE_NAMES", "KEYS", "reconstruction_dict", "save_reconstruction", "load_reconstruction",
           "result_dict"]

# modality -> (file name, object key, auxiliary key, scan key)
KEYS = {
    "conventional": ("reconstruction.pt", "sample", "probe", "positions_xy"),
    "fourier": ("fpm_reconstruction.pt", "object", "pupil", "led_indices_xy"),
    "coded": ("coded_reconstruction.pt", "object", "coded_surface", "shifts_xy_pixels"),
    "nearfield": ("coded_reconstruction.pt", "object", "coded_surface", "shifts_xy_pixels"),
}
FILE_NAMES = {m: k[0] for m, k in KEYS.items()}


def _cpu(x, dtype=None) -> torch.Tensor:
    t = x.detach() if torch.is_tensor(x) else torch.from_numpy(np.ascontiguousarray(x))
    t = t.cpu()
    return t if dtype is None else t.to(dtype)


def reconstruction_dict(modality: str, obj, aux, scan, observed_amplitude, args: dict | None = None) -> dict:
    """The reference's dictionary for ``modality``.

    ``obj`` / ``aux``: complex object and probe / pupil / coded surface; ``scan``: int64
    positions or LED corners, or the shifts in pixels (coded: ``shifts_xy * n``, as the
    reference stores ``shifts_px``); ``observed_amplitude``: float32 amplitudes
    ``sqrt(scale * counts)``; ``args``: the run's settings (the reference stores its argparse
    namespace as a dict).
    """
    if modality not in KEYS:
        raise ValueError(f"modality must be one of {sorted(KEYS)}, got {modality!r}")
    _, k_obj, k_aux, k_scan = KEYS[modality]
    return {
        k_obj: _cpu(obj, torch.complex64),
        k_aux: _cpu(aux, torch.complex64),
        k_scan: _cpu(scan),
        "observed_amplitude": _cpu(observed_amplitude, torch.float32),
        "args": dict(args or {}),
    }


def save_reconstruction(out_dir, modality: str, obj, aux, scan, observed_amplitude,
                        args: dict | None = None) -> Path:
    """Write ``out_dir / FILE_NAMES[modality]``; returns the path."""
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    path = out / FILE_NAMES[modality]
    torch.save(reconstruction_dict(modality, obj, aux, scan, observed_amplitude, args), path)
    return path


def load_reconstruction(path) -> tuple[str, dict]:
    """Read a reconstruction file; returns ``(modality, dict)``.  The modality is told by the
    auxiliary key (``probe`` / ``pupil`` / ``coded_surface``; coded and near-field share a
    format and load as ``"coded"``)."""
    d = torch.load(Path(path), map_location="cpu", weights_only=False)
    for modality in ("conventional", "fourier", "coded"):
        _, k_obj, k_aux, k_scan = KEYS[modality]
        if k_aux in d and k_obj in d:
            return modality, d
    raise ValueError(f"{path}: not a reconstruction file (keys {sorted(d)})")


def result_dict(request, result, args: dict | None = None) -> dict:
    """The reference dictionary for one served reconstruction (``serving.ReconRequest`` and its
    ``ReconResult``): final object and auxiliary, the request's scan and its observed
    amplitudes."""
    meas = np.asarray(request.meas).astype(np.float32)
    observed = np.sqrt(meas * np.float32(request.scale))
    scan = request.pos
    if request.modality in ("coded", "nearfield"):
        scan = np.asarray(request.pos, dtype=np.float32) * np.float32(np.asarray(request.obj0).shape[-1])
    info = {"rid": request.rid, "iters": request.iters, "final_loss": result.final_loss}
    info.update(args or {})
    return reconstruction_dict(request.modality, result.obj, result.aux, scan, observed, info)
