"""Device-side window checks of the conventional operators, reported without a host sync.

The conventional kernels check every scan window on the device: a window that leaves the
object is skipped and bit 0 of the workspace status word is set (``ptx_workspace_status``).
Positions that arrive as host tensors are checked on the host before the launch (no device
round trip).  For device-resident positions -- the reference's training loop indexes a
device tensor of positions every step (``train_ptychography.py:549``) -- three modes:

* ``"deferred"`` (default): after the launch the status word is copied in stream order into a
  page-locked slot and an event is recorded; the next call of any conventional operator on
  that device (or :func:`check_errors`) raises ``ValueError`` for every earlier call whose
  copy has completed with the bit set.  No host synchronisation, no host copy of positions.
* ``"sync"``: the same copy, waited for at once, so the offending call itself raises.
* ``"host"``: the positions are copied to the host and checked before the launch (one
  device-to-host synchronisation per call).

Calls made while a stream is being captured into a CUDA graph are not tracked.
"""

from __future__ import annotations

import threading
from collections import deque

import torch

from . import _abi

_MODES = ("deferred", "sync", "host")
_mode = "deferred"
_lock = threading.Lock()
_pending: deque = deque()  # (device index, event, slot index, what)
_slots: dict[int, torch.Tensor] = {}  # device -> pinned uint32 ring
_next_slot: dict[int, int] = {}
_RING = 256


def set_bounds_check(mode: str) -> None:
    """Select how out-of-object windows of device-resident positions are reported:
    ``"deferred"`` (default), ``"sync"`` or ``"host"`` (see the module docstring)."""
    global _mode
    if mode not in _MODES:
        raise ValueError(f"bounds check mode must be one of {_MODES}, got {mode!r}")
    _mode = mode


def bounds_check_mode() -> str:
    return _mode


def _raise_for(what: str) -> None:
    raise ValueError(f"{what}: a scan window leaves the object (its frame was skipped); "
                     "positions must satisfy 0 <= x <= W - pw and 0 <= y <= H - ph.")


def _slot(dev: int) -> tuple[torch.Tensor, int]:
    ring = _slots.get(dev)
    if ring is None:
        ring = torch.zeros(_RING, dtype=torch.int32).pin_memory()
        _slots[dev] = ring
        _next_slot[dev] = 0
    k = _next_slot[dev]
    _next_slot[dev] = (k + 1) % _RING
    return ring, k


def _drain(block: bool, device: int | None = None) -> None:
    """Retire pending checks in order (all, or those of `device`); raise for the first failure.
    With block=False stop at the first check whose copy has not completed."""
    failed = None
    with _lock:
        keep = deque()
        while _pending:
            dev, ev, k, what = _pending.popleft()
            if device is not None and dev != device:
                keep.append((dev, ev, k, what))
                continue
            if not ev.query():
                if not block:
                    keep.append((dev, ev, k, what))
                    keep.extend(e for e in _pending)
                    _pending.clear()
                    break
                ev.synchronize()
            if failed is None and int(_slots[dev][k]) & 1:
                failed = what
        _pending.extend(keep)
    if failed is not None:
        _raise_for(failed)


def check_errors(block: bool = True) -> None:
    """Raise ``ValueError`` if an earlier conventional call with device positions met a window
    outside the object (waits for their status copies when ``block``)."""
    _drain(block)


def before_call(device: torch.device) -> None:
    """Report completed failures of earlier calls on `device` (non-blocking)."""
    if _pending:
        _drain(False, device.index)


def after_call(workspace: torch.Tensor, device: torch.device, what: str) -> None:
    """Queue the status copy of the call that just used `workspace` (device positions only)."""
    stream = torch.cuda.current_stream(device)
    with torch.cuda.device(device):
        if torch.cuda.is_current_stream_capturing():
            return
    dev = device.index if device.index is not None else torch.cuda.current_device()
    if len(_pending) >= _RING - 1:
        _drain(True)
    with _lock:
        ring, k = _slot(dev)
        ring[k] = 0
        _abi.call("ptx_workspace_status", workspace.data_ptr(), ring.data_ptr() + 4 * k, stream.cuda_stream)
        ev = torch.cuda.Event()
        ev.record(stream)
        _pending.append((dev, ev, k, what))
    if _mode == "sync":
        _drain(True, dev)
