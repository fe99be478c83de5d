"""ctypes binding of libptychox (the C ABI declared in ``include/ptychox.h``).

The library is loaded from ``ptychox_b200/_lib/libptychox.so``.  There is no CPU
fallback: if the library is missing or cannot be loaded every operator raises.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libptychox.so"

PTX_OK = 0
PTX_ERR_INVALID_ARGUMENT = 1
PTX_ERR_UNSUPPORTED_SIZE = 2
PTX_ERR_WORKSPACE = 3
PTX_ERR_CUDA = 4
PTX_ERR_OUT_OF_BOUNDS = 5
PTX_ERR_TIMEOUT = 6

PTX_MODALITY_CONVENTIONAL = 0
PTX_MODALITY_FOURIER = 1
PTX_MODALITY_CODED = 2
PTX_MODALITY_NEARFIELD = 3

PTX_CONSTRAIN_NONE = 0
PTX_CONSTRAIN_UNIT_AMPLITUDE = 1
PTX_CONSTRAIN_REAL_NONNEGATIVE = 2

_p = C.c_void_p
_i = C.c_int
_f = C.c_float
_sz = C.c_size_t

# name -> (restype, argtypes); mirrors include/ptychox.h
SIGNATURES: dict[str, tuple] = {
    "ptx_version": (_i, []),
    "ptx_last_error": (C.c_char_p, []),
    "ptx_clear_cache": (_i, []),
    "ptx_launch_count": (C.c_longlong, []),
    "ptx_set_units_per_cta": (_i, [_i]),
    "ptx_set_thread_units_per_cta": (_i, [_i]),
    "ptx_get_units_per_cta": (_i, []),
    "ptx_stage_host_bytes": (_i, [_p, _p, _sz, _p]),
    "ptx_profile_enable": (_i, [_i]),
    "ptx_profile_reset": (_i, []),
    "ptx_profile_kinds": (_i, []),
    "ptx_profile_read": (_i, [_i, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "ptx_profile_name": (C.c_char_p, [_i]),
    "ptx_fft_supported": (_i, [_i]),
    "ptx_fft_engine": (_i, [_i]),
    "ptx_fft_prepare": (_i, [_i]),
    "ptx_base_workspace_bytes": (_sz, [_i, _i, _i]),
    "ptx_base_forward": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _p, _p, _sz, _p]),
    "ptx_base_backward": (_i, [_p, _p, _p, _i, _i, _p, _i, _i, _p, _i, _p, _p, _p, _sz, _p]),
    "ptx_base_sweep": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _f, _p, _p, _p, _p, _sz, _p]),
    "ptx_base_sweep_small": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _f, _p, _p, _p, _p, _sz, _p]),
    "ptx_base_subpix_workspace_bytes": (_sz, [_i, _i, _i]),
    "ptx_base_subpix_forward": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _p, _p, _sz, _p]),
    "ptx_base_subpix_backward": (_i, [_p, _p, _p, _i, _i, _p, _i, _i, _p, _i, _p, _p, _p, _sz, _p]),
    "ptx_base_subpix_sweep": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _f, _p, _p, _p, _p, _sz, _p]),
    "ptx_fpm_workspace_bytes": (_sz, [_i, _i, _i, _i, _i]),
    "ptx_fpm_forward": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _p, _p, _p, _sz, _p]),
    "ptx_fpm_backward": (_i, [_p, _p, _p, _i, _i, _p, _i, _i, _p, _i, _p, _p, _p, _sz, _p]),
    "ptx_fpm_sweep": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _f, _p, _p, _p, _p, _sz, _p]),
    "ptx_coded_workspace_bytes": (_sz, [_i, _i]),
    "ptx_coded_forward": (_i, [_p, _p, _p, _p, _i, _p, _i, _i, _p, _p, _p, _p, _sz, _p]),
    "ptx_coded_backward": (_i, [_p, _p, _p, _p, _p, _p, _p, _i, _p, _i, _i, _p, _p, _p, _sz, _p]),
    "ptx_coded_sweep": (_i, [_p, _p, _p, _p, _i, _p, _i, _i, _p, _f, _p, _p, _p, _p, _sz, _p]),
    "ptx_coded_fd_workspace_bytes": (_sz, [_i, _i, _i]),
    "ptx_coded_sweep_fd": (_i, [_p, _p, _p, _p, _i, _p, _i, _i, _p, _f, _i, _p, _p, _p, _p, _sz, _p]),
    "ptx_coded_sweep_ex_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "ptx_coded_sweep_ex": (_i, [_p, _p, _p, _p, _i, _p, _i, _i, _p, _f, _i, _p, _p, _p, _p, _p, _sz, _p]),
    "ptx_adam_step": (_i, [_p, _p, _p, _p, _sz, _p, _f, _f, _f, _f, _i, _p]),
    "ptx_base_sweep_noalloc": (_i, [_p, _i, _i, _p, _i, _i, _p, _i, _p, _f, _p, _p, _p, _p]),
    "ptx_workspace_status": (_i, [_p, _p, _p]),
    "ptx_status_code": (_i, [C.c_uint]),
    "ptx_reg_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "ptx_reg_upsampled_peak": (_i, [_p, _i, _i, _i, _i, _p, _p, _p, _p, _p, _sz, _p]),
    "ptx_server_create": (_i, [_i, _sz, _i, _p]),
    "ptx_server_submit": (_i, [_p, _p, _p]),
    "ptx_server_poll": (_i, [_p, C.c_longlong, _p, _p, _p, _p, _p]),
    "ptx_server_poll_ex": (_i, [_p, C.c_longlong, _p, _p, _p, _p, _p, _p]),
    "ptx_server_destroy": (_i, [_p]),
}

_lock = threading.Lock()
_lib = None


class PtychoXError(RuntimeError):
    """A libptychox call failed (CUDA error, workspace, device-wait timeout)."""


def lib_path() -> Path:
    return _LIB_PATH


def load() -> C.CDLL:
    """Load libptychox once; raise if it is absent (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not _LIB_PATH.exists():
            raise ImportError(
                f"libptychox is not built ({_LIB_PATH}); run `python -m ptychox_b200.build` "
                "(the sm_100a library is the only implementation)"
            )
        lib = C.CDLL(str(_LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().ptx_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str) -> None:
    """Map a status code to the exception type the reference raises for that failure."""
    if status == PTX_OK:
        return
    msg = f"{what}: {last_error()}"
    if status in (PTX_ERR_INVALID_ARGUMENT, PTX_ERR_UNSUPPORTED_SIZE, PTX_ERR_OUT_OF_BOUNDS):
        raise ValueError(msg)
    raise PtychoXError(msg)


def call(name: str, *args) -> None:
    fn = getattr(load(), name)
    check(fn(*args), name)


def query(name: str, *args):
    return getattr(load(), name)(*args)


def profile_read() -> dict[str, tuple[float, int]]:
    """``{kernel name: (total ms, timed launches)}`` of the event profiler (synchronises)."""
    lib = load()
    out = {}
    for k in range(lib.ptx_profile_kinds()):
        ms = C.c_double(0.0)
        n = C.c_longlong(0)
        check(lib.ptx_profile_read(k, C.byref(ms), C.byref(n)), "ptx_profile_read")
        if n.value:
            out[lib.ptx_profile_name(k).decode()] = (ms.value, n.value)
    return out
