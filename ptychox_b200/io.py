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

The MATLAB near-field example keeps its measurements in ``imgRawData.mat``
(``matlab/Examples/Near-field Ptychography/gen_img.m:59``: ``imRaw`` ``[pix, pix, n]``
intensities, ``ScanPos`` ``[n, 2]`` ``(locX, locY)`` in low-resolution pixels, ``pattern``
the complex probe field on the ``mag``-times finer grid, ``env`` the struct of
``+helpers/init_expEnvs.m``).  ``save_matlab_dataset`` / ``load_matlab_dataset`` write and
read that file (MATLAB v5 format through scipy.io), and ``nearfield_inputs`` turns it into
this library's near-field arguments the way ``fdpr_recon_cuda.m:10-18,65`` prepares them.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import torch

__all__ = ["FILE_NAMES", "KEYS", "reconstruction_dict", "save_reconstruction", "load_reconstruction",
           "result_dict", "save_matlab_dataset", "load_matlab_dataset", "nearfield_inputs"]

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


def _np(x) -> np.ndarray:
    return x.detach().cpu().numpy() if torch.is_tensor(x) else np.asarray(x)


def save_matlab_dataset(path, im_raw, scan_pos, pattern, env: dict | None = None) -> Path:
    """Write ``imgRawData.mat`` as ``gen_img.m:59`` saves it.

    ``im_raw``: ``[n, h, w]`` intensities (stored MATLAB-style as ``imRaw`` ``[h, w, n]``);
    ``scan_pos``: ``[n, 2]`` ``(locX, locY)`` in low-resolution pixels; ``pattern``: complex
    ``[H, W]`` probe field (single precision, as the script's ``gpuArray(single(...))``);
    ``env``: the experiment struct (field name -> array or scalar), empty when ``None``.
    """
    from scipy.io import savemat

    raw = np.ascontiguousarray(np.transpose(_np(im_raw).astype(np.float64), (1, 2, 0)))
    mdict = {
        "imRaw": raw,
        "ScanPos": _np(scan_pos).astype(np.float64).reshape(-1, 2),
        "pattern": _np(pattern).astype(np.complex64),
        "env": {k: _np(v) for k, v in (env or {}).items()},
    }
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    savemat(str(path), mdict, do_compression=False)
    return path


def load_matlab_dataset(path) -> dict:
    """Read an ``imgRawData.mat`` (written by ``gen_img.m`` or :func:`save_matlab_dataset`).

    Returns ``{"im_raw": [n, h, w] float64, "scan_pos": [n, 2] float64, "pattern": complex
    [H, W], "env": dict}`` (``imRaw`` moved from MATLAB's ``[h, w, n]`` to ``[n, h, w]``)."""
    from scipy.io import loadmat

    d = loadmat(str(path), squeeze_me=False, struct_as_record=False)
    raw = np.asarray(d["imRaw"])
    if raw.ndim == 2:  # a single image: MATLAB drops the trailing singleton
        raw = raw[:, :, None]
    env = {}
    if "env" in d:
        e = d["env"]
        e = e[0, 0] if isinstance(e, np.ndarray) and e.size == 1 else e
        for name in getattr(e, "_fieldnames", []) or []:
            v = getattr(e, name)
            env[name] = np.squeeze(v) if np.asarray(v).size == 1 else np.asarray(v)
    return {"im_raw": np.ascontiguousarray(np.transpose(raw, (2, 0, 1))).astype(np.float64),
            "scan_pos": np.asarray(d["ScanPos"], dtype=np.float64).reshape(-1, 2),
            "pattern": np.asarray(d["pattern"]),
            "env": env}


def nearfield_inputs(dataset: dict, max_count: int = 65535) -> dict:
    """Near-field arguments from a loaded ``imgRawData.mat``, as ``fdpr_recon_cuda.m`` prepares
    them: the raw images shifted to a zero minimum and scaled (``:12-14``), the shifts in
    units of the low-resolution side, ``ScanPos / pix`` (``:65``; the field side is
    ``mag * pix``, so this is the shift in field pixels over the field side, the library's
    ``shifts_xy``), and the downsampling factor ``mag``.

    The fused losses take uint16 counts: ``counts = round(I / scale)`` with ``scale`` mapping
    the largest intensity to ``max_count`` (a quantisation of the float images); the observed
    amplitude is then ``sqrt(scale * counts)``."""
    raw = np.asarray(dataset["im_raw"], dtype=np.float64)
    raw = raw - raw.min()
    top = raw.max()
    if top > 0:
        raw = raw / top
    n, h, w = raw.shape
    field = np.asarray(dataset["pattern"])
    if field.shape[0] % h or field.shape[1] % w or field.shape[0] // h != field.shape[1] // w:
        raise ValueError(f"pattern {field.shape} is not a whole multiple of the {h}x{w} images")
    scale = float(np.float32(1.0 / max_count))
    counts = np.rint(raw / scale).clip(0, max_count).astype(np.uint16)
    return {"shifts_xy": (np.asarray(dataset["scan_pos"], dtype=np.float64) / h).astype(np.float32),
            "downsample": field.shape[0] // h, "probe_field": field.astype(np.complex64),
            "measured": counts, "scale": scale, "intensity": raw.astype(np.float32)}
