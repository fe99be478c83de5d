"""The native reconstruction server (``ptx_server_*`` in libptychox) from Python.

Same requests and results as ``ptychox_b200.serving`` (``ReconRequest`` / ``ReconResult``):
the scheduling, admission, resident state, CUDA-graph capture and replay run in the
library's own scheduler thread, so a host process (or another language through the C ABI)
submits reconstructions and polls for them without driving the GPU itself.
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _abi
from .optim import CONSTRAINTS
from .serving import ReconRequest, ReconResult

__all__ = ["PtxReconRequest", "NativeReconstructionServer", "ReplicaServer"]

_MODALITY = {
    "conventional": _abi.PTX_MODALITY_CONVENTIONAL,
    "fourier": _abi.PTX_MODALITY_FOURIER,
    "coded": _abi.PTX_MODALITY_CODED,
    "nearfield": _abi.PTX_MODALITY_NEARFIELD,
}


class PtxReconRequest(C.Structure):
    """``ptx_recon_request`` of ``include/ptychox.h``."""

    _fields_ = [
        ("modality", C.c_int), ("obj_h", C.c_int), ("obj_w", C.c_int), ("aux_h", C.c_int), ("aux_w", C.c_int),
        ("batch", C.c_int), ("downsample", C.c_int), ("iters", C.c_int), ("scale", C.c_float),
        ("lr_obj", C.c_float), ("lr_aux", C.c_float), ("constrain_obj", C.c_int), ("constrain_aux", C.c_int),
        ("obj0", C.c_void_p), ("aux0", C.c_void_p), ("scan", C.c_void_p), ("measured", C.c_void_p),
        ("transfer_1", C.c_void_p), ("transfer_2", C.c_void_p), ("target_ratio", C.c_float),
    ]


def _host(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=dtype)


class NativeReconstructionServer:
    """``ptx_server_create`` on ``device``; ``hbm_budget`` 0 = 70% of the free memory."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_active: int = 8):
        _abi.load()
        self._h = C.c_void_p()
        _abi.call("ptx_server_create", int(device), int(hbm_budget), int(max_active), C.addressof(self._h))
        self._shapes: dict[int, tuple] = {}

    def submit(self, req: ReconRequest) -> int:
        """Queue ``req`` (copied at the call); returns the server's id for it."""
        coded = req.modality in ("coded", "nearfield")
        obj = _host(req.obj0, np.complex64)
        aux = _host(req.aux0, np.complex64)
        scan = _host(req.pos, np.float32 if coded else np.int64)
        meas = _host(req.meas, np.uint16)
        t1 = None if req.t1 is None else _host(req.t1, np.complex64)
        t2 = None if req.t2 is None else _host(req.t2, np.complex64)
        d = PtxReconRequest(
            modality=_MODALITY[req.modality], obj_h=obj.shape[0], obj_w=obj.shape[1], aux_h=aux.shape[0],
            aux_w=aux.shape[1], batch=int(scan.shape[0]), downsample=int(req.ds), iters=int(req.iters),
            scale=float(req.scale), lr_obj=float(req.lrs[0]), lr_aux=float(req.lrs[1]),
            constrain_obj=CONSTRAINTS[req.constraints[0]], constrain_aux=CONSTRAINTS[req.constraints[1]],
            obj0=obj.ctypes.data, aux0=aux.ctypes.data, scan=scan.ctypes.data, measured=meas.ctypes.data,
            transfer_1=None if t1 is None else t1.ctypes.data, transfer_2=None if t2 is None else t2.ctypes.data,
            target_ratio=float(req.target_ratio or 0.0))
        rid = C.c_longlong(0)
        _abi.call("ptx_server_submit", self._h, C.addressof(d), C.addressof(rid))
        self._shapes[rid.value] = (req, obj.shape, aux.shape)
        return rid.value

    def poll(self, rid: int) -> ReconResult | None:
        """The result of ``rid`` once finished (then forgotten by the server), else None."""
        if rid not in self._shapes:  # the library reports the unknown id (ValueError)
            done = C.c_int(0)
            _abi.call("ptx_server_poll", self._h, C.c_longlong(rid), C.addressof(done), None, None, None, None)
        req, so, sa = self._shapes[rid]
        obj = np.empty(so, np.complex64)
        aux = np.empty(sa, np.complex64)
        done, loss, lat, iters = C.c_int(0), C.c_double(0.0), C.c_double(0.0), C.c_int(0)
        try:
            _abi.call("ptx_server_poll_ex", self._h, C.c_longlong(rid), C.addressof(done), C.addressof(loss),
                      C.addressof(lat), C.addressof(iters), obj.ctypes.data, aux.ctypes.data)
        except Exception:
            del self._shapes[rid]
            raise
        if not done.value:
            return None
        del self._shapes[rid]
        return ReconResult(req.rid, req.modality, req.arrival, admitted=0.0, finished=req.arrival + lat.value,
                           final_loss=loss.value, obj=obj, aux=aux, sweeps=int(iters.value))

    def run(self, requests: list[ReconRequest], poll_interval: float = 1e-3) -> list[ReconResult]:
        """Submit all ``requests`` now and wait for them; results in ``rid`` order."""
        ids = {self.submit(r): r.rid for r in requests}
        out = {}
        while ids:
            for sid in list(ids):
                res = self.poll(sid)
                if res is not None:
                    out[ids.pop(sid)] = res
            if ids:
                time.sleep(poll_interval)
        return [out[k] for k in sorted(out)]

    def close(self) -> None:
        if self._h:
            _abi.call("ptx_server_destroy", self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReplicaServer:
    """Serving replicas: one native server per device in ``devices`` (a device may repeat),
    each request pinned to the replica with the fewest outstanding requests; no
    communication between replicas (the multi-GPU mode of the reconstruction service)."""

    def __init__(self, devices, hbm_budget: int = 0, max_active: int = 8):
        self.replicas = [NativeReconstructionServer(int(d), hbm_budget, max_active) for d in devices]
        self._where: dict[int, tuple[int, int]] = {}  # our id -> (replica, its id)
        self._outstanding = [0] * len(self.replicas)
        self._next = 1

    def submit(self, req: ReconRequest) -> int:
        k = min(range(len(self.replicas)), key=lambda i: (self._outstanding[i], i))
        sid = self.replicas[k].submit(req)
        rid = self._next
        self._next += 1
        self._where[rid] = (k, sid)
        self._outstanding[k] += 1
        return rid

    def replica_of(self, rid: int) -> int:
        return self._where[rid][0]

    def poll(self, rid: int) -> ReconResult | None:
        k, sid = self._where[rid]
        try:
            res = self.replicas[k].poll(sid)
        except Exception:
            del self._where[rid]
            self._outstanding[k] -= 1
            raise
        if res is not None:
            del self._where[rid]
            self._outstanding[k] -= 1
        return res

    def run(self, requests: list[ReconRequest], poll_interval: float = 1e-3) -> list[ReconResult]:
        """Submit all ``requests`` now and wait for them; results in ``rid`` order."""
        ids = {self.submit(r): r.rid for r in requests}
        out = {}
        while ids:
            for sid in list(ids):
                res = self.poll(sid)
                if res is not None:
                    out[ids.pop(sid)] = res
            if ids:
                time.sleep(poll_interval)
        return [out[k] for k in sorted(out)]

    def close(self) -> None:
        for r in self.replicas:
            r.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
