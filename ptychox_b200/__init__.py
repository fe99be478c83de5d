"""ptychox_b200 — B200-native (sm_100a) PtychoX operators behind the reference's API.

Drop-in for ``python/ptychoX`` (``__init__.py:1-27`` of THUHoloLab/PtychoX): the same
operator names, aliases and cache hooks, backed by ``libptychox`` (C ABI in
``include/ptychox.h``).  Added: fused forward+loss+adjoint sweeps (``*_loss``).
"""

from ._status import bounds_check_mode, check_errors, set_bounds_check
from ._utils import matlab_positions_to_torch
from .base import clear_cuda_plan_cache as clear_base_cuda_plan_cache
from .base import (
    ptychoX_base,
    ptychoX_base_loss,
    ptychoX_base_subpixel,
    ptychoX_base_subpixel_loss,
    ptychography_base,
)
from .coded import clear_cuda_plan_cache as clear_coded_cuda_plan_cache
from .coded import (
    coded_ptychography,
    nearfield_ptychography,
    ptychoX_coded,
    ptychoX_coded_loss,
    ptychoX_nearfield,
    ptychoX_nearfield_loss,
)
from .fpm import clear_cuda_plan_cache as clear_fpm_cuda_plan_cache
from .fpm import fourier_ptychography, ptychoX_fourier, ptychoX_fourier_loss


def clear_cuda_plan_cache() -> None:
    """Drop cached FFT plans of every modality (one shared library cache)."""
    clear_base_cuda_plan_cache()
    clear_fpm_cuda_plan_cache()
    clear_coded_cuda_plan_cache()


__all__ = [
    "clear_cuda_plan_cache",
    "clear_base_cuda_plan_cache",
    "clear_fpm_cuda_plan_cache",
    "clear_coded_cuda_plan_cache",
    "ptychoX_coded",
    "ptychoX_coded_loss",
    "coded_ptychography",
    "ptychoX_nearfield",
    "ptychoX_nearfield_loss",
    "nearfield_ptychography",
    "ptychoX_fourier",
    "ptychoX_fourier_loss",
    "fourier_ptychography",
    "ptychoX_base",
    "ptychoX_base_loss",
    "ptychoX_base_subpixel",
    "ptychoX_base_subpixel_loss",
    "ptychography_base",
    "matlab_positions_to_torch",
    "set_bounds_check",
    "bounds_check_mode",
    "check_errors",
]
