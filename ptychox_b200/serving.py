"""Continuous-batching reconstruction server on one GPU.

Reconstructions of mixed modality and size arrive over time.  The server

* admits them in arrival order while the sum of their resident bytes fits an HBM budget
  (object, probe / pupil / mask, gradients, Adam moments, counts, scan, workspace);
* keeps each admitted reconstruction's state resident until its last iteration;
* captures one iteration -- fused sweep (forward, amplitude-MSE loss, adjoint) plus the
  Adam steps -- as a CUDA graph per reconstruction, once, at admission;
* every scheduler tick replays the next iteration of every active reconstruction on its
  own stream, so iterations of different reconstructions overlap on the device, and
  reconstructions join as soon as earlier ones finish and free their memory;
* stops a reconstruction at a fixed error when its request asks for one: each replay copies
  its sweep loss to page-locked memory, and once a completed iteration's loss is at most
  ``target_ratio`` times the initial loss no further iteration is queued;
* reports per-request latency (arrival to final state on the host), p50 / p99, and
  sweeps/s.

``run_plain`` solves the same requests one at a time with the unfused operator API and
``torch.optim.Adam`` -- the reference drivers' training loop (``train_ptychography.py``
:529-560) -- as the baseline.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch
import torch.nn.functional as F

from . import _abi
from ._utils import ptr
from .base import use_small_sweep
from .optim import FusedAdam

__all__ = ["ReconRequest", "ReconResult", "ReconstructionServer", "run_plain", "percentile"]

MODALITIES = ("conventional", "fourier", "coded", "nearfield")


@dataclass
class ReconRequest:
    """One reconstruction: host arrays plus its schedule.

    ``obj0`` / ``aux0``: initial object and probe (conventional) / pupil (fourier) /
    coded surface or probe field (coded, near-field); ``pos``: int64 positions / LED
    corners or float32 shifts; ``meas``: uint16 counts; ``t1`` / ``t2``: transfer
    functions (coded; ``t1`` None for near-field); ``ds``: downsample.
    """

    rid: int
    modality: str
    arrival: float
    obj0: np.ndarray
    aux0: np.ndarray
    pos: np.ndarray
    meas: np.ndarray
    scale: float
    iters: int = 50
    lrs: tuple = (0.02, 0.02)
    constraints: tuple = (None, None)
    t1: np.ndarray | None = None
    t2: np.ndarray | None = None
    ds: int = 1
    # stop at a fixed error: once an iteration's loss is at most target_ratio times the initial
    # loss (the sweep at obj0 / aux0) no further iteration runs; 0 runs all `iters`
    target_ratio: float = 0.0

    def units(self) -> int:
        return int(self.pos.shape[0])


@dataclass
class ReconResult:
    rid: int
    modality: str
    arrival: float
    admitted: float = 0.0
    finished: float = 0.0
    final_loss: float = float("nan")
    obj: np.ndarray | None = None
    aux: np.ndarray | None = None
    sweeps: int = 0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def percentile(values, q: float) -> float:
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if len(values) else float("nan")


def _workspace_bytes(req: ReconRequest, cap: int) -> int:
    n_obj = req.obj0.shape
    b = req.units()
    if req.modality == "conventional":
        ph, pw = req.aux0.shape
        frame = math.ceil(pw / 16) * 16 * ph * 8
        full = _abi.query("ptx_base_workspace_bytes", ph, pw, b)
        return int(min(full, max(256 + frame, cap)))
    if req.modality == "fourier":
        lh, lw = req.aux0.shape
        full = _abi.query("ptx_fpm_workspace_bytes", n_obj[0], n_obj[1], lh, lw, b)
        fixed = _abi.query("ptx_fpm_workspace_bytes", n_obj[0], n_obj[1], lh, lw, 1)
        return int(min(full, max(fixed, cap)))
    n = n_obj[0]
    full = _abi.query("ptx_coded_workspace_bytes", n, b)
    fixed = _abi.query("ptx_coded_workspace_bytes", n, 1)
    return int(min(full, max(fixed, cap)))


def request_bytes(req: ReconRequest, ws_cap: int) -> int:
    """Resident device bytes of one admitted reconstruction."""
    params = (req.obj0.size + req.aux0.size) * 8
    state = params * 4  # gradients (1x) + Adam moments (2x) + copy of the parameters at launch (1x slack)
    extra = req.meas.nbytes + req.pos.nbytes
    if req.t1 is not None:
        extra += req.t1.nbytes
    if req.t2 is not None:
        extra += req.t2.nbytes
    return int(params + state + extra + _workspace_bytes(req, ws_cap) + 4096)


class _Slot:
    """Resident state of one admitted reconstruction and its captured iteration."""

    def __init__(self, req: ReconRequest, dev: torch.device, ws_cap: int, use_graph: bool, priority: int = 0):
        self.req = req
        self.dev = dev
        self.stream = torch.cuda.Stream(device=dev, priority=priority)
        self.iters_launched = 0
        self.bytes = request_bytes(req, ws_cap)
        with torch.cuda.stream(self.stream):
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev, non_blocking=True)  # noqa: E731
            self.obj = t(req.obj0)
            self.aux = t(req.aux0)
            self.pos = t(req.pos)
            self.meas = t(req.meas)
            self.t1 = None if req.t1 is None else t(req.t1)
            self.t2 = None if req.t2 is None else t(req.t2)
            self.g_obj = torch.empty_like(self.obj)
            self.g_aux = torch.empty_like(self.aux)
            self.loss = torch.zeros((), dtype=torch.float64, device=dev)
            self.ws = torch.empty(_workspace_bytes(req, ws_cap), dtype=torch.uint8, device=dev)
            self.adam = FusedAdam([self.obj, self.aux], list(req.lrs), constraints=list(req.constraints))
        self.stream_handle = self.stream.cuda_stream
        self.graph = None
        self.limit = req.iters  # iterations to run (fewer once the error target is met)
        self.loss_host = torch.full((), float("nan"), dtype=torch.float64).pin_memory()
        # the warm-up sweep (FFT plans and kernel attributes, outside any capture) runs at
        # obj0 / aux0: its loss is the initial loss the error target is relative to
        with torch.cuda.stream(self.stream):
            self._sweep()
        self.stream.synchronize()
        self.target = float(req.target_ratio) * float(self.loss.item()) if req.target_ratio > 0 else -1.0
        if use_graph:
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.stream(self.stream):
                self.graph.capture_begin(capture_error_mode="relaxed")
                try:
                    self._iterate()
                finally:
                    self.graph.capture_end()
        self.done = torch.cuda.Event()
        self.inflight: list[torch.cuda.Event] = []

    def _sweep(self) -> None:
        r = self.req
        s = self.stream_handle
        if r.modality == "conventional":
            (h, w), (ph, pw) = self.obj.shape, self.aux.shape
            entry = "ptx_base_sweep_small" if use_small_sweep(ph, pw, r.units()) else "ptx_base_sweep"
            _abi.call(entry, ptr(self.obj), h, w, ptr(self.aux), ph, pw, ptr(self.pos), r.units(),
                      ptr(self.meas), float(r.scale), ptr(self.loss), ptr(self.g_obj), ptr(self.g_aux), ptr(self.ws),
                      self.ws.numel(), s)
        elif r.modality == "fourier":
            (h, w), (lh, lw) = self.obj.shape, self.aux.shape
            _abi.call("ptx_fpm_sweep", ptr(self.obj), h, w, ptr(self.aux), lh, lw, ptr(self.pos), r.units(),
                      ptr(self.meas), float(r.scale), ptr(self.loss), ptr(self.g_obj), ptr(self.g_aux), ptr(self.ws),
                      self.ws.numel(), s)
        else:
            _abi.call("ptx_coded_sweep", ptr(self.obj), ptr(self.aux), ptr(self.t1), ptr(self.t2), self.obj.shape[0],
                      ptr(self.pos), r.units(), int(r.ds), ptr(self.meas), float(r.scale), ptr(self.loss),
                      ptr(self.g_obj), ptr(self.g_aux), ptr(self.ws), self.ws.numel(), s)

    def _iterate(self) -> None:
        self._sweep()
        self.adam.step([self.g_obj, self.g_aux])
        if self.target >= 0.0:
            self.loss_host.copy_(self.loss, non_blocking=True)

    def launch_next(self, max_inflight: int) -> None:
        """Queue the next iteration unless ``max_inflight`` of this slot's are still queued, the
        schedule is complete, or a completed iteration met the error target."""
        completed = False
        while self.inflight and self.inflight[0].query():
            self.inflight.pop(0)
            completed = True
        if completed and self.target >= 0.0 and self.iters_launched < self.limit:
            if float(self.loss_host) <= self.target:
                self.limit = self.iters_launched
                self.done.record(self.stream)
        if self.iters_launched >= self.limit or len(self.inflight) >= max_inflight:
            return
        with torch.cuda.stream(self.stream):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._iterate()
        self.iters_launched += 1
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.inflight.append(ev)
        if self.iters_launched == self.limit:
            self.done.record(self.stream)

    def finished(self) -> bool:
        return self.iters_launched == self.limit and self.done.query()


class ReconstructionServer:
    """Admit by HBM budget, keep state resident, replay captured iterations concurrently."""

    def __init__(self, device: torch.device | str = "cuda", hbm_budget: int | None = None,
                 max_active: int = 8, workspace_cap: int = 512 << 20, use_graphs: bool = True,
                 max_inflight: int = 2, units_per_cta: int = 8):
        self.dev = torch.device(device)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget = int(free * 0.7)
        self.budget = int(hbm_budget)
        self.max_active = max_active
        self.ws_cap = int(workspace_cap)
        self.use_graphs = use_graphs
        self.max_inflight = max_inflight
        # persistent passes of concurrent reconstructions must interleave CTA by CTA
        self.units_per_cta = int(units_per_cta)

    def run(self, requests: list[ReconRequest], realtime: bool = True) -> list[ReconResult]:
        """Serve ``requests`` (arrival times in seconds from the start); returns results in rid order."""
        _abi.load()
        # the bound covers this thread's launches and captures only (process-wide setting kept)
        _abi.query("ptx_set_thread_units_per_cta", self.units_per_cta)
        try:
            return self._run(requests, realtime)
        finally:
            _abi.query("ptx_set_thread_units_per_cta", -1)

    def _run(self, requests: list[ReconRequest], realtime: bool) -> list[ReconResult]:
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in pending:
            if request_bytes(r, self.ws_cap) > self.budget:
                raise ValueError(f"request {r.rid} needs more than the HBM budget ({self.budget} bytes)")
        results = {r.rid: ReconResult(r.rid, r.modality, r.arrival) for r in pending}
        active: list[_Slot] = []
        used = 0
        t0 = time.perf_counter()
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: float("inf"))
        while pending or active:
            now = clock()
            # admission: FIFO, arrived, within budget and slot count
            while pending and pending[0].arrival <= now and len(active) < self.max_active:
                nxt = pending[0]
                need = request_bytes(nxt, self.ws_cap)
                if used + need > self.budget and active:
                    break
                pending.pop(0)
                # older reconstructions get higher stream priority (the GPU prefers their CTAs)
                low, high = torch.cuda.Stream.priority_range()
                prio = max(high, min(low, high + len(active)))
                slot = _Slot(nxt, self.dev, self.ws_cap, self.use_graphs, priority=prio)
                used += slot.bytes
                active.append(slot)
                results[nxt.rid].admitted = clock() if realtime else 0.0
            # one iteration per active reconstruction per tick (bounded queue depth per stream)
            for slot in active:
                slot.launch_next(self.max_inflight)
            # retire finished reconstructions
            still = []
            for slot in active:
                if slot.finished():
                    res = results[slot.req.rid]
                    res.final_loss = float(slot.loss.item())
                    res.obj = slot.obj.cpu().numpy()
                    res.aux = slot.aux.cpu().numpy()
                    res.sweeps = slot.iters_launched
                    res.finished = clock() if realtime else 0.0
                    used -= slot.bytes
                    slot.graph = None
                else:
                    still.append(slot)
            active = still
            if not active and pending and realtime:
                wait = pending[0].arrival - clock()
                if wait > 0:
                    time.sleep(min(wait, 0.05))
        torch.cuda.synchronize(self.dev)
        return [results[k] for k in sorted(results)]


def run_plain(requests: list[ReconRequest], device: torch.device | str = "cuda",
              realtime: bool = True) -> list[ReconResult]:
    """Solve the requests one at a time with the unfused operators and torch.optim.Adam."""
    from . import ptychoX_base, ptychoX_coded, ptychoX_fourier, ptychoX_nearfield

    dev = torch.device(device)
    t0 = time.perf_counter()
    out = []
    for req in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        if realtime:
            wait = req.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        res = ReconResult(req.rid, req.modality, req.arrival, admitted=time.perf_counter() - t0)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        obj = t(req.obj0).requires_grad_(True)
        aux = t(req.aux0).requires_grad_(True)
        pos = t(req.pos)
        observed = torch.sqrt(t(req.meas).to(torch.float32) * np.float32(req.scale))
        t1 = None if req.t1 is None else t(req.t1)
        t2 = None if req.t2 is None else t(req.t2)
        opt = torch.optim.Adam([{"params": [obj], "lr": req.lrs[0]}, {"params": [aux], "lr": req.lrs[1]}],
                               betas=(0.9, 0.999), eps=1e-16)
        loss = None
        target = -1.0
        done_iters = 0
        for it in range(req.iters):
            if req.modality == "conventional":
                pred = ptychoX_base(obj, aux, pos)
            elif req.modality == "fourier":
                pred = ptychoX_fourier(obj, aux, pos)
            elif req.modality == "coded":
                pred = ptychoX_coded(obj, aux, t1, t2, pos, req.ds)
            else:
                pred = ptychoX_nearfield(obj, aux, t2, pos, req.ds)
            loss = F.mse_loss(pred, observed)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            done_iters = it + 1
            with torch.no_grad():
                for p, c in ((obj, req.constraints[0]), (aux, req.constraints[1])):
                    if c == "unit_amplitude":
                        a = p.abs()
                        p.copy_(torch.where(a > 1, p / a.clamp_min(1e-30), p))
                    elif c == "real_nonnegative":
                        p.copy_(p.real.clamp_min(0.0).to(torch.complex64))
            if req.target_ratio > 0:  # the reference loop reads every loss (train_ptychography.py:560)
                value = float(loss.item())
                if it == 0:
                    target = float(req.target_ratio) * value
                if value <= target:
                    break
        res.final_loss = float(loss.item())
        res.obj = obj.detach().cpu().numpy()
        res.aux = aux.detach().cpu().numpy()
        res.sweeps = done_iters
        res.finished = time.perf_counter() - t0
        out.append(res)
    return sorted(out, key=lambda r: r.rid)


# ---------------------------------------------------------------------------------------
# request synthesis (seeded; measurements from this library's forward operators)
# ---------------------------------------------------------------------------------------

_SMOOTH = sorted({2 ** a * 3 ** b * 5 ** c for a in range(11) for b in range(3) for c in range(3)
                  if 16 <= 2 ** a * 3 ** b * 5 ** c <= 1024})


def snap_smooth(n: float) -> int:
    """Nearest 2^a 3^b 5^c transform length in [16, 1024]."""
    return min(_SMOOTH, key=lambda m: (abs(m - n), m))


def snap_pow2(n: float) -> int:
    """Nearest power-of-two transform length in [16, 1024] (ties round up)."""
    return min((2 ** a for a in range(4, 11)), key=lambda m: (abs(math.log2(m) - math.log2(n)), -m))


def synthesize_request(rid: int, modality: str, arrival: float, size: dict, seed: int, device,
                       iters: int = 50, target_ratio: float = 0.0) -> ReconRequest:
    """One seeded reconstruction problem; counts from the forward model of the truth.

    ``size``: conventional {"p", "grid", "step", "n"}; fourier {"n", "h", "grid"};
    coded / near-field {"n", "count", "ds"}.  The object starts flat (0.9); the probe /
    pupil / mask starts at the truth times a small random phase error.
    """
    from . import ptychoX_base, ptychoX_coded, ptychoX_fourier, ptychoX_nearfield, synth

    rng = np.random.default_rng(seed)
    dev = torch.device(device)
    t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    t1 = t2 = None
    ds = 1
    if modality == "conventional":
        p, grid, step, n = size["p"], size["grid"], size["step"], size["n"]
        truth = synth.random_object(n, n, rng)
        aux_true = synth.gaussian_probe(p, p, rng)
        pos = synth.raster_positions(grid, step, 8, 2, rng)
        with torch.no_grad():
            amp = ptychoX_base(t(truth), t(aux_true), t(pos))
        photons, per_pixel, brightest = 1e4 * (p / 128.0) ** 2, False, False
        lrs, cons = (0.02, 0.002), ("unit_amplitude", None)
    elif modality == "fourier":
        n, h, grid = size["n"], size["h"], size["grid"]
        truth = synth.random_object(n, n, rng)
        aux_true = synth.circular_pupil(h, 0.3)
        dx = synth.fpm_dx_for_pupil(n, h, 0.1, 0.532, 0.3)
        pos = synth.fpm_led_windows(n, h, grid, 4.0, 90.0, 0.532, dx)
        with torch.no_grad():
            amp = ptychoX_fourier(t(truth), t(aux_true), t(pos))
        photons, per_pixel, brightest = 5e3, True, True
        lrs, cons = (2.0, 0.002), (None, None)
    else:
        n, count, ds = size["n"], size["count"], size["ds"]
        truth = synth.random_object(n, n, rng)
        aux_true = synth.binary_mask(n, 0.5, rng)
        t2 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 2e-3)
        t1 = None if modality == "nearfield" else synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 396.95e-6)
        pos = synth.coded_shifts(count, 20.0 * n / 1024.0, n, rng)
        with torch.no_grad():
            if modality == "nearfield":
                amp = ptychoX_nearfield(t(truth), t(aux_true), t(t2), t(pos), ds)
            else:
                amp = ptychoX_coded(t(truth), t(aux_true), t(t1), t(t2), t(pos), ds)
        photons, per_pixel, brightest = 2e3, True, False
        lrs, cons = (0.02, 0.002), ("unit_amplitude", "real_nonnegative")
    inten = amp.double() ** 2
    sums = inten.flatten(1).sum(dim=1)
    per = float(sums.max() if brightest else sums.mean())
    scale = float(np.float32(per / (photons * (inten[0].numel() if per_pixel else 1))))
    gen = torch.Generator(device=dev).manual_seed(seed)
    counts = torch.poisson(inten / scale, generator=gen).clamp_max(65535).to(torch.int32).to(torch.uint16)
    obj0 = np.full(truth.shape, 0.9, dtype=np.complex64)
    aux0 = (aux_true * np.exp(0.05j * rng.standard_normal(aux_true.shape))).astype(np.complex64)
    return ReconRequest(rid=rid, modality=modality, arrival=float(arrival), obj0=obj0, aux0=aux0, pos=pos,
                        meas=counts.cpu().numpy(), scale=scale, iters=iters, lrs=lrs, constraints=cons, t1=t1,
                        t2=t2, ds=ds, target_ratio=float(target_ratio))


def serving_mix(n_requests: int, seed: int = 0, rate: float = 20.0) -> list[tuple]:
    """Arrivals and sizes of the mixed stream: ``(rid, modality, arrival, size)``.

    Poisson arrivals at ``rate`` per second; 40 / 30 / 20 / 10 % drawn from the
    conventional small scan (128^2 probe, 11x11 raster), Fourier (256^2 pupil, 15x15
    LEDs, 1024^2 spectrum), coded / near-field (1024^2 field, 64 shifts, ds 4) and the
    conventional large scan (512^2 probe, 30x30 raster), sizes jittered by U[0.75, 1.25]:
    conventional probe sides snapped to the nearest 2^a 3^b 5^c length (96..640: lengths
    such as 100, 120, 144, 160, 480, 600 run on the mixed-radix register FFT), scan grids
    jittered with positions held in [49, 900]; Fourier pupil sides snapped likewise
    (192..320) in a spectrum of the largest smooth side up to min(1024, 4 h), LED grids
    jittered; coded / near-field fields snapped to the nearest smooth side in [768, 1024] that
    the downsampling factor 4 divides (768, 800, 864, 900, 960, 972, 1000, 1024), shift counts
    jittered.
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        u = float(rng.uniform())
        j = lambda: float(rng.uniform(0.75, 1.25))  # noqa: E731
        if u < 0.4 or u >= 0.9:
            big = u >= 0.9
            p0, g0, s0 = (512, 30, 48) if big else (128, 11, 32)
            p = snap_smooth(p0 * j())
            grid = int(min(30, max(7, round(g0 * j()))))
            step = max(4, int(round(s0 * p / p0)))
            n = 8 + (grid - 1) * step + p + 4 + 8
            n = int(math.ceil(n / 16) * 16)
            out.append((rid, "conventional", t, {"p": p, "grid": grid, "step": step, "n": n}))
        elif u < 0.7:
            grid = int(min(15, max(7, round(15 * j()))))
            h = snap_smooth(256 * j())
            n = max(m for m in _SMOOTH if m <= min(1024, 4 * h))
            out.append((rid, "fourier", t, {"n": n, "h": h, "grid": grid}))
        else:
            count = int(max(16, round(64 * j())))
            n0 = 1024 * j()
            n = min((m for m in _SMOOTH if 768 <= m <= 1024 and m % 4 == 0), key=lambda m: (abs(m - n0), m))
            out.append((rid, "coded" if rng.uniform() < 0.5 else "nearfield", t, {"n": n, "count": count, "ds": 4}))
    return out
