"""Benchmark of the fused forward+adjoint ptychography sweep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

One *step* is one sweep: forward, amplitude-MSE loss against uint16 counts and adjoint
over every scan position of one reconstruction, producing the FP64 loss and the object
and probe gradients.  The default workload is the conventional configuration
900 positions x 512x512 probe -> 2048x2048 object.  Inputs are seeded synthetic data.

Our arm prints one JSON line (rank 0) with ``value`` = sweeps/s over all ranks from
device-resident inputs (CUDA events per step, L2 flushed between steps, max over
ranks), ``e2e`` = the same through the public API with host buffers, ``roofline`` of
the sweep, ``cpu_baseline`` (CPU oracle on this host, bounded sample), ``clocks``.
``--impl reference`` times the reference's own PyTorch CPU path (the unmodified
``ptychoX`` package installed in ``baseline/_ref`` by ``baseline/install_reference.sh``:
the operator with ``use_cuda_kernels=False`` in complex64, ``F.mse_loss`` and
``.backward()``) on all host cores, one whole sweep per step; without that install it
falls back to the oracle's numpy restatement (``kind: "port"``).

With N > 1 (torchrun) the ranks share one reconstruction: each sweeps its row band of the
scan and the weighted loss and gradients are all-reduced over NCCL (strong scaling; the
weak figure, every rank sweeping all positions, is reported beside it).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


# ---------------------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------------------

def hbm_peak() -> tuple[float, str]:
    try:
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Workload:
    """One benchmark configuration: synthesis, fused sweep, public-API step, byte model."""

    name = ""
    units = "positions"

    def metric(self) -> str:
        raise NotImplementedError

    def bytes_per_sweep(self) -> float:
        raise NotImplementedError

    def config(self) -> dict:
        raise NotImplementedError


class Conventional(Workload):
    """Raster-scanned conventional ptychography (configs 0 and 1)."""

    def __init__(self, name, n_obj, p, grid, step, origin, jitter, photons):
        self.name, self.n_obj, self.p = name, n_obj, p
        self.grid, self.step, self.origin, self.jitter, self.photons = grid, step, origin, jitter, photons
        self.batch = grid * grid

    def metric(self):
        return f"fwd+adj sweeps/s ({self.batch}×{self.p}²→{self.n_obj}²)"

    def bytes_per_sweep(self):
        # per position 8 P^2 gather + 2 P^2 counts + 16 P^2 grad_O RMW; + 16 P^2 + 8 N^2 per sweep
        p2 = float(self.p) ** 2
        return 26.0 * p2 * self.batch + 16.0 * p2 + 8.0 * float(self.n_obj) ** 2

    def config(self):
        return {"workload": self.name, "modality": "conventional", "positions": self.batch,
                "probe": [self.p, self.p], "object": [self.n_obj, self.n_obj],
                "raster": f"{self.grid}x{self.grid} step {self.step} origin {self.origin} jitter U[-{self.jitter},{self.jitter}]",
                "photons_per_pattern": self.photons}

    def host(self, seed):
        from ptychox_b200 import synth

        rng = np.random.default_rng(seed)
        obj = synth.random_object(self.n_obj, self.n_obj, rng)
        probe = synth.gaussian_probe(self.p, self.p, rng)
        pos = synth.raster_positions(self.grid, self.step, self.origin, self.jitter, rng)
        guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
        return {"truth": obj, "obj": guess, "aux": probe, "pos": pos}

    def synth(self, seed, dev):
        import torch

        from ptychox_b200 import ptychoX_base

        h = self.host(seed)
        with torch.no_grad():
            amp = ptychoX_base(torch.from_numpy(h["truth"]).to(dev), torch.from_numpy(h["aux"]).to(dev),
                               torch.from_numpy(h["pos"]).to(dev))
            meas, scale = device_poisson(amp, self.photons, seed, per_pixel=False)
        return self._pack(h, meas, scale, dev)

    def _pack(self, h, meas, scale, dev):
        import torch

        return {"obj": torch.from_numpy(h["obj"]).to(dev), "aux": torch.from_numpy(h["aux"]).to(dev),
                "pos": torch.from_numpy(h["pos"]).to(dev), "meas": meas, "scale": scale, "host": h}

    def workspace(self, prob, dev):
        from ptychox_b200 import _abi
        from ptychox_b200._utils import workspace

        return workspace(_abi.query("ptx_base_workspace_bytes", self.p, self.p, self.batch), dev)

    def sweep(self, prob, ws):
        from ptychox_b200.base import base_sweep

        return base_sweep(prob["obj"], prob["aux"], prob["pos"], prob["meas"], prob["scale"], ws=ws)

    def loss_api(self, obj, aux, pos, prob):
        from ptychox_b200 import ptychoX_base_loss

        return ptychoX_base_loss(obj, aux, pos, prob["meas"], prob["scale"])

    def cpu_sweep(self, h, meas, scale, k, workers):
        from oracle import ptycho_oracle as O

        O.base_sweep(h["obj"], h["aux"], h["pos"][:k], meas[:k], scale, fp64=False, workers=workers)


class ConventionalSubpixel(Conventional):
    """Conventional ptychography at sub-pixel scan positions: config 1's raster with its
    U[-3, 3] jitter kept real (float64 positions), the five-pass sub-pixel sweep."""

    def metric(self):
        return f"fwd+adj sweeps/s ({self.batch}×{self.p}²→{self.n_obj}², sub-pixel positions)"

    def config(self):
        c = super().config()
        c["modality"] = "conventional, sub-pixel positions (Fourier-shifted windows)"
        c["raster"] = c["raster"] + " (real-valued)"
        return c

    def host(self, seed):
        from ptychox_b200 import synth

        rng = np.random.default_rng(seed)
        obj = synth.random_object(self.n_obj, self.n_obj, rng)
        probe = synth.gaussian_probe(self.p, self.p, rng)
        pos = synth.raster_positions_subpixel(self.grid, self.step, self.origin, float(self.jitter), rng)
        guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
        return {"truth": obj, "obj": guess, "aux": probe, "pos": pos}

    def synth(self, seed, dev):
        import torch

        from ptychox_b200 import ptychoX_base_subpixel

        h = self.host(seed)
        with torch.no_grad():
            amp = ptychoX_base_subpixel(torch.from_numpy(h["truth"]).to(dev), torch.from_numpy(h["aux"]).to(dev),
                                        torch.from_numpy(h["pos"]).to(dev))
            meas, scale = device_poisson(amp, self.photons, seed, per_pixel=False)
        return self._pack(h, meas, scale, dev)

    def workspace(self, prob, dev):
        from ptychox_b200 import _abi
        from ptychox_b200._utils import workspace

        return workspace(_abi.query("ptx_base_subpix_workspace_bytes", self.p, self.p, self.batch), dev)

    def sweep(self, prob, ws):
        from ptychox_b200.base import base_subpixel_sweep

        return base_subpixel_sweep(prob["obj"], prob["aux"], prob["pos"], prob["meas"], prob["scale"], ws=ws)

    def loss_api(self, obj, aux, pos, prob):
        from ptychox_b200 import ptychoX_base_subpixel_loss

        return ptychoX_base_subpixel_loss(obj, aux, pos, prob["meas"], prob["scale"])

    def cpu_sweep(self, h, meas, scale, k, workers):
        from oracle import ptycho_oracle as O

        O.base_subpix_sweep(h["obj"], h["aux"], h["pos"][:k], meas[:k], scale, fp64=False, workers=workers)


class Fourier(Conventional):
    """Fourier ptychography (config 2): 15x15 LEDs, 256^2 pupil, 1024^2 spectrum."""

    def __init__(self, name, n, h, grid, photons):
        self.name, self.n_obj, self.p, self.grid, self.photons = name, n, h, grid, photons
        self.batch = grid * grid

    def metric(self):
        return f"fwd+adj sweeps/s (FPM {self.batch}×{self.p}²←{self.n_obj}²)"

    def bytes_per_sweep(self):
        # per LED 26 h^2; per sweep + 72 N^2 (spectrum and gradient transforms) + 16 h^2
        h2 = float(self.p) ** 2
        return 26.0 * h2 * self.batch + 72.0 * float(self.n_obj) ** 2 + 16.0 * h2

    def config(self):
        return {"workload": self.name, "modality": "fourier", "leds": self.batch, "pupil": [self.p, self.p],
                "object": [self.n_obj, self.n_obj], "na": 0.1, "wavelength_um": 0.532, "led_pitch_mm": 4.0,
                "led_height_mm": 90.0, "photons_per_pixel_brightest": self.photons}

    def host(self, seed):
        from ptychox_b200 import synth

        rng = np.random.default_rng(seed)
        obj = synth.random_object(self.n_obj, self.n_obj, rng)
        pupil = synth.circular_pupil(self.p, 0.3)
        dx = synth.fpm_dx_for_pupil(self.n_obj, self.p, 0.1, 0.532, 0.3)
        led = synth.fpm_led_windows(self.n_obj, self.p, self.grid, 4.0, 90.0, 0.532, dx)
        guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
        return {"truth": obj, "obj": guess, "aux": pupil, "pos": led}

    def synth(self, seed, dev):
        import torch

        from ptychox_b200 import ptychoX_fourier

        h = self.host(seed)
        with torch.no_grad():
            amp = ptychoX_fourier(torch.from_numpy(h["truth"]).to(dev), torch.from_numpy(h["aux"]).to(dev),
                                  torch.from_numpy(h["pos"]).to(dev))
            meas, scale = device_poisson(amp, self.photons, seed, per_pixel=True, brightest=True)
        return self._pack(h, meas, scale, dev)

    def workspace(self, prob, dev):
        from ptychox_b200 import _abi
        from ptychox_b200._utils import workspace

        return workspace(_abi.query("ptx_fpm_workspace_bytes", self.n_obj, self.n_obj, self.p, self.p, self.batch),
                         dev)

    def sweep(self, prob, ws):
        from ptychox_b200.fpm import fpm_sweep

        return fpm_sweep(prob["obj"], prob["aux"], prob["pos"], prob["meas"], prob["scale"], ws=ws)

    def loss_api(self, obj, aux, pos, prob):
        from ptychox_b200 import ptychoX_fourier_loss

        return ptychoX_fourier_loss(obj, aux, pos, prob["meas"], prob["scale"])

    def cpu_sweep(self, h, meas, scale, k, workers):
        from oracle import ptycho_oracle as O

        O.fpm_sweep(h["obj"], h["aux"], h["pos"][:k], meas[:k], scale, fp64=False, workers=workers)


class Coded(Conventional):
    """Coded / near-field ptychography (config 3): 1024^2 field, 64 shifts, ds 4."""

    def __init__(self, name, n, count, ds, photons, nearfield, loss="mse"):
        self.name, self.n_obj, self.batch, self.ds, self.photons = name, n, count, ds, photons
        self.nearfield = nearfield
        self.loss = loss  # "mse" or train_coded.py's fd_loss ("fd-isotropic" / "fd-anisotropic")
        self.p = n

    def metric(self):
        kind = "near-field" if self.nearfield else "coded"
        tail = "" if self.loss == "mse" else f", {self.loss} loss"
        return f"fwd+adj sweeps/s ({kind} {self.batch}×{self.n_obj}², ds {self.ds}{tail})"

    def bytes_per_sweep(self):
        n2 = float(self.n_obj) ** 2
        return 240.125 * n2 * self.batch + 64.0 * n2

    def config(self):
        return {"workload": self.name, "modality": "near-field" if self.nearfield else "coded", "loss": self.loss,
                "positions": self.batch, "field": [self.n_obj, self.n_obj], "downsample": self.ds,
                "pixel_um": 1.85, "wavelength_um": 0.5, "z_mm": 2.0,
                "z1_um": None if self.nearfield else 396.95, "mask": "binary 50% fill",
                "shifts_px": "U[-20, 20]", "photons_per_pixel": self.photons}

    def host(self, seed):
        from ptychox_b200 import synth

        rng = np.random.default_rng(seed)
        n = self.n_obj
        obj = synth.random_object(n, n, rng)
        mask = synth.binary_mask(n, 0.5, rng)
        t2 = synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 2e-3)
        t1 = None if self.nearfield else synth.angular_spectrum_transfer(n, 1.85e-6, 0.5e-6, 396.95e-6)
        shifts = synth.coded_shifts(self.batch, 20.0, n, rng)
        guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
        return {"truth": obj, "obj": guess, "aux": mask, "pos": shifts, "t1": t1, "t2": t2}

    def synth(self, seed, dev):
        import torch

        from ptychox_b200 import ptychoX_coded, ptychoX_nearfield

        h = self.host(seed)
        t = lambda a: None if a is None else torch.from_numpy(a).to(dev)  # noqa: E731
        with torch.no_grad():
            if self.nearfield:
                amp = ptychoX_nearfield(t(h["truth"]), t(h["aux"]), t(h["t2"]), t(h["pos"]), self.ds)
            else:
                amp = ptychoX_coded(t(h["truth"]), t(h["aux"]), t(h["t1"]), t(h["t2"]), t(h["pos"]), self.ds)
            meas, scale = device_poisson(amp, self.photons, seed, per_pixel=True)
        prob = self._pack(h, meas, scale, dev)
        prob["t1"], prob["t2"] = t(h["t1"]), t(h["t2"])
        return prob

    def workspace(self, prob, dev):
        from ptychox_b200 import _abi
        from ptychox_b200._utils import workspace

        if self.loss != "mse":
            return workspace(_abi.query("ptx_coded_fd_workspace_bytes", self.n_obj, self.batch, self.ds), dev)
        return workspace(_abi.query("ptx_coded_workspace_bytes", self.n_obj, self.batch), dev)

    def sweep(self, prob, ws):
        from ptychox_b200.coded import coded_sweep

        return coded_sweep(prob["obj"], prob["aux"], prob["t1"], prob["t2"], prob["pos"], self.ds, prob["meas"],
                           prob["scale"], ws=ws, loss=self.loss)

    def loss_api(self, obj, aux, pos, prob):
        from ptychox_b200 import ptychoX_coded_loss, ptychoX_nearfield_loss

        if self.nearfield:
            return ptychoX_nearfield_loss(obj, aux, prob["t2"], pos, self.ds, prob["meas"], prob["scale"],
                                          loss=self.loss)
        return ptychoX_coded_loss(obj, aux, prob["t1"], prob["t2"], pos, self.ds, prob["meas"], prob["scale"],
                                  loss=self.loss)

    def cpu_sweep(self, h, meas, scale, k, workers):
        from oracle import ptycho_oracle as O

        O.coded_sweep(h["obj"], h["aux"], h["t1"], h["t2"], h["pos"][:k], self.ds, meas[:k], scale, fp64=False,
                      workers=workers, loss=self.loss)


WORKLOADS = {
    w.name: w
    for w in [
        Conventional("conventional-900x512-2048", 2048, 512, 30, 48, 64, 3, 1e5),
        Conventional("conventional-121x128-512", 512, 128, 11, 32, 8, 2, 1e4),
        ConventionalSubpixel("conventional-subpixel-900x512-2048", 2048, 512, 30, 48, 64, 3, 1e5),
        # {2,3,5}-smooth probe sides of the serving mix's range, on the mixed-radix FFT kernels
        Conventional("conventional-121x96-512", 512, 96, 11, 32, 8, 2, 1e4),
        Conventional("conventional-121x160-640", 640, 160, 11, 40, 8, 2, 1e4),
        Conventional("conventional-400x640-2048", 2048, 640, 20, 64, 64, 3, 1e5),
        Fourier("fourier-225x256-1024", 1024, 256, 15, 5e3),
        # config 2 and 3 geometry at smooth sides that are not powers of two (mixed-radix kernels)
        Fourier("fourier-169x240-960", 960, 240, 13, 5e3),
        Coded("coded-64x1024-ds4", 1024, 64, 4, 2e3, nearfield=False),
        Coded("coded-64x960-ds4", 960, 64, 4, 2e3, nearfield=False),
        Coded("nearfield-64x1024-ds4", 1024, 64, 4, 2e3, nearfield=True),
        Coded("coded-fd-64x1024-ds4", 1024, 64, 4, 2e3, nearfield=False, loss="fd-isotropic"),
    ]
}
DEFAULT_WORKLOAD = "conventional-900x512-2048"


def device_poisson(amp, photons, seed, per_pixel=False, brightest=False):
    """uint16 Poisson counts of amp^2 / scale on the device (``synth.poisson_counts_device``)."""
    from ptychox_b200.synth import poisson_counts_device

    return poisson_counts_device(amp, photons, seed, per_pixel=per_pixel, brightest=brightest)


# ---------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of all kernels of one sweep, from
# the ncu captures summarised in profiles/ (the same scope as `achieved`: one whole sweep).
MEASURED_TRAFFIC = {
    "conventional-900x512-2048": (7.319e9, "profiles/base_sweep_kernels_96positions_full.md",
                                  "96-position capture scaled by 900/96"),
    "fourier-225x256-1024": (0.4366e9, "profiles/fpm_sweep_225x256_full.md",
                             "full-size captures, one per kernel"),
    "coded-64x1024-ds4": (6.60e9, "profiles/coded_sweep_16x1024_full.md", "16-shift capture scaled by 64/16"),
}


def subset(wl: Workload, k: int) -> Workload:
    """The same workload on its first k scan units (positions, LEDs or shifts), for small
    profiling cases; the JSON line records the subset in its config."""
    import copy

    w = copy.copy(wl)
    full_host = wl.host

    def host(seed):
        h = full_host(seed)
        h["pos"] = h["pos"][:k]
        return h

    w.host = host
    w.batch = min(k, wl.batch)
    full_config = wl.config

    def config():
        c = full_config()
        c["units_subset"] = w.batch
        return c

    w.config = config
    return w


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from ptychox_b200 import _abi

    wl = WORKLOADS[args.workload]
    if args.units:
        wl = subset(wl, args.units)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    _abi.load()

    # Every rank synthesises the same problem.  Strong scaling (default with N > 1): the ranks
    # share one reconstruction, each sweeping its row band of the scan (shard_positions) and
    # all-reducing the weighted loss and gradients, so a step is one whole sweep.  Weak: every
    # rank sweeps all units and the results are averaged (N sweeps per step).
    from ptychox_b200.distributed import reduce_sweep, shard_positions

    strong = world > 1 and args.scaling == "strong"
    prob = wl.synth(seed=1000, dev=dev)
    full_prob = prob
    local_units, total_units = wl.batch, wl.batch * (1 if strong else world)
    if strong:
        idx = shard_positions(prob["host"]["pos"], rank, world)
        it = torch.from_numpy(idx).to(dev)
        prob = dict(prob, pos=prob["pos"][it].contiguous(), meas=prob["meas"][it].contiguous(),
                    host=dict(prob["host"], pos=np.ascontiguousarray(prob["host"]["pos"][idx])))
        local_units = len(idx)
    ws = wl.workspace(full_prob, dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        loss, g_obj, g_aux = wl.sweep(prob, ws)
        if world > 1:  # data-parallel sweep: global mean over all ranks' units
            reduce_sweep(loss, [g_obj, g_aux], local_units, total_units)
        return loss, g_obj, g_aux

    def timed(k: int, fn) -> list[float]:
        pairs = []
        stream = torch.cuda.current_stream(dev)
        for _ in range(k):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            flush.zero_()  # write > L2 between timed steps (outside the events)
            pairs.append((a, b))
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in pairs]

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    clocks = ClockSampler(local)
    clocks.start()  # sampling runs from the warm-up through the timed region (200 ms period)
    time.sleep(0.5)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    # ---- timed region -------------------------------------------------------------
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = _abi.query("ptx_launch_count")
    step_ms = timed(args.steps, step)
    launches = _abi.query("ptx_launch_count") - launches0
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms))
    ms_per_step = total_ms / args.steps
    value = (1 if strong else world) * args.steps / (total_ms / 1e3)

    multi = None
    if world > 1:
        # the sharded sweep equals the whole sweep on one GPU (checked on rank 0, no collective)
        loss_r, go_r, ga_r = step()
        torch.cuda.synchronize(dev)
        multi = {"mode": "strong" if strong else "weak", "units_per_rank": local_units}
        if strong and rank == 0:
            loss_1, go_1, ga_1 = wl.sweep(full_prob, ws)
            torch.cuda.synchronize(dev)
            multi["parity_vs_one_gpu"] = {
                "loss": abs(float(loss_r) - float(loss_1)) / abs(float(loss_1)),
                "grad_obj": float((go_r - go_1).norm() / go_1.norm()),
                "grad_aux": float((ga_r - ga_1).norm() / ga_1.norm())}
        if strong:
            # the weak figure beside it: every rank sweeps all units of the same problem

            def weak_step():
                loss, g_obj, g_aux = wl.sweep(full_prob, ws)
                reduce_sweep(loss, [g_obj, g_aux], wl.batch, wl.batch * world)

            dist.barrier()
            weak_ms = max_over_ranks(sum(timed(args.steps, weak_step)))
            multi["weak"] = {"value": world * args.steps / (weak_ms / 1e3), "unit": "sweeps/s",
                             "ms_per_step": weak_ms / args.steps}

    # ---- roofline: the sweep's kernels timed with library events ------------------
    _abi.query("ptx_profile_reset")
    _abi.query("ptx_profile_enable", 1)
    prof_ms = timed(args.steps, step)
    _abi.query("ptx_profile_enable", 0)
    per_kernel = _abi.profile_read()
    peak, peak_kind = hbm_peak()
    sweep_bytes = wl.bytes_per_sweep()
    # per GPU: the share of the sweep this rank moves in one step
    achieved = sweep_bytes * (local_units / wl.batch) / (ms_per_step / 1e3) / 1e9
    kern_total = sum(v[0] for v in per_kernel.values()) or 1.0
    kernels = [{"name": k, "launches_per_step": n / args.steps, "ms_per_launch": ms / n, "share": ms / kern_total}
               for k, (ms, n) in sorted(per_kernel.items(), key=lambda kv: -kv[1][0])]
    roofline = {
        "bound": "hbm",
        "achieved": achieved,
        "peak": peak,
        "unit": "GB/s",
        "frac": achieved / peak,
        "traffic": None if args.units else MEASURED_TRAFFIC.get(wl.name, (None,))[0],
        "traffic_source": None if args.units else MEASURED_TRAFFIC.get(wl.name, (None, None, None))[1:],
        "peak_kind": f"{peak_kind} hbm_gbs (of {peak_kind})",
        "scope": "fused sweep: all passes of one sweep on one stream, algorithmic bytes per sweep / sweep time",
        "algorithmic_bytes_per_sweep": sweep_bytes,
        "profiled_sweep_ms": statistics.median(prof_ms),
        "kernels": kernels,
    }

    # ---- e2e: public API with pinned host buffers -----------------------------------
    # A training loop as a user writes it against the public API, with each step's inputs
    # uploaded from pinned host memory and its loss and gradients read back.  The copies run on
    # two copy streams with double-buffered device inputs, so step k+1's upload and step k-1's
    # read-back overlap step k's sweep (PCIe is full duplex).  Timed from the first upload to
    # the last read-back on the device.
    host = prob["host"]
    h_obj = torch.from_numpy(host["obj"]).pin_memory()
    h_aux = torch.from_numpy(host["aux"]).pin_memory()
    h_pos = torch.from_numpy(host["pos"]).pin_memory()
    out_go = [torch.empty_like(h_obj).pin_memory() for _ in range(2)]
    out_ga = [torch.empty_like(h_aux).pin_memory() for _ in range(2)]
    out_loss = [torch.empty((), dtype=torch.float64).pin_memory() for _ in range(2)]
    d_in = [(torch.empty_like(h_obj, device=dev), torch.empty_like(h_aux, device=dev)) for _ in range(2)]
    s_comp = torch.cuda.current_stream(dev)
    s_up = torch.cuda.Stream(device=dev)
    s_down = torch.cuda.Stream(device=dev)

    def upload(b):
        with torch.cuda.stream(s_up):
            for d, h in zip(d_in[b], (h_obj, h_aux)):
                d.copy_(h, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s_up)
        return ev

    def e2e_run(k: int) -> float:
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(s_up)
        ready = [upload(0), None]
        freed = [None, None]  # the compute stream is done with buffer b
        for i in range(k):
            b = i & 1
            s_comp.wait_event(ready[b])
            d_obj = d_in[b][0].detach().requires_grad_(True)
            d_aux = d_in[b][1].detach().requires_grad_(True)
            # the scan goes in as pinned host memory: the API checks it on the host and uploads it
            loss = wl.loss_api(d_obj, d_aux, h_pos, prob)
            loss.backward()
            g_obj, g_aux, l_det = d_obj.grad, d_aux.grad, loss.detach()
            if world > 1:
                reduce_sweep(l_det, [g_obj, g_aux], local_units, total_units)
            done = torch.cuda.Event()
            done.record(s_comp)
            freed[b] = done
            # the next step's upload is queued after this step's own (small) scan upload, so the
            # scan copy never waits behind it on the copy engine
            if i + 1 < k:
                if freed[b ^ 1] is not None:
                    s_up.wait_event(freed[b ^ 1])
                ready[b ^ 1] = upload(b ^ 1)
            s_down.wait_event(done)
            with torch.cuda.stream(s_down):
                out_go[b].copy_(g_obj, non_blocking=True)
                out_ga[b].copy_(g_aux, non_blocking=True)
                out_loss[b].copy_(l_det, non_blocking=True)
            for t in (g_obj, g_aux, l_det):
                t.record_stream(s_down)  # keep the memory until the read-back has finished
        s_up.wait_stream(s_down)
        s_up.wait_stream(s_comp)
        end.record(s_up)
        torch.cuda.synchronize(dev)
        return start.elapsed_time(end)

    e2e_run(max(2, args.warmup))
    if world > 1:
        dist.barrier()
    e2e_ms = max_over_ranks(e2e_run(args.steps))
    h2d = (h_obj.numel() + h_aux.numel()) * 8 + h_pos.numel() * h_pos.element_size()
    d2h = (out_go[0].numel() + out_ga[0].numel()) * 8 + 8
    e2e = {"value": (1 if strong else world) * args.steps / (e2e_ms / 1e3), "unit": "sweeps/s",
           "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h,
           "note": "public loss API (autograd); each step uploads object, probe/pupil/mask and scan from pinned "
                   "host memory (the scan through the API's own pinned upload) and reads back the loss and "
                   "both gradients, on two copy streams with double-buffered inputs (uploads and read-backs "
                   "overlap the neighbouring steps' sweeps); "
                   "measured counts resident in HBM (uploaded once, as the reference training loop keeps "
                   "observed amplitudes on the device); timed from the first upload to the last read-back"}

    # ---- CPU baseline (rank 0, N = 1) --------------------------------------------------
    cpu = cpu_port = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        meas_host = prob["meas"].cpu().numpy()
        cpu = cpu_reference_rate(wl, host, meas_host, prob["scale"], budget_s=args.cpu_budget)
        # the oracle's numpy restatement (secondary figure; the primary one when the reference
        # install is absent)
        cpu_port = cpu_sample_rate(wl, host, meas_host, prob["scale"], budget_s=args.cpu_budget / 2)
        if cpu is None:
            cpu, cpu_port = cpu_port, None
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu_rates(wl, host, prob["meas"].cpu().numpy(), prob["scale"], dev, flush)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving and not args.units and wl.name == DEFAULT_WORKLOAD:
        serving = serving_record(args, dev)

    if rank == 0:
        cfg = wl.config()
        cfg["parallelism"] = ((f"dp{world}: one reconstruction, row-band position shards, NCCL all-reduce of the "
                               f"weighted loss and gradients" if strong else
                               f"dp{world}: every rank sweeps all positions, NCCL all-reduce")
                              if world > 1 else "single GPU")
        cfg["l2"] = "flushed between timed steps (256 MB write outside the step events)"
        line = {
            "metric": wl.metric(),
            "value": value,
            "unit": "sweeps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "strong" if strong else "weak",
            "vs_baseline": None,
            "dtype": "c64 (FP32 FFT/constraint, FP64 loss sum)",
            "data": "synthetic (seeded object and scan, Poisson uint16 counts from the forward model)",
            "config": cfg,
            "multi_gpu": multi,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "cpu_baseline_port": cpu_port,
            "reference_gpu": ref_gpu,
            "serving": serving,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


REF_DIR = ROOT / "baseline" / "_ref"


def reference_package():
    """The reference's own ``ptychoX`` package as installed in ``baseline/_ref`` (None when absent).

    ``baseline/install_reference.sh`` pip-installs the unmodified reference there (its CUDA
    extension built from source for sm_100a) together with its driver scripts, which hold
    ``fd_loss`` (``train_coded.py:101-107``)."""
    if not (REF_DIR / "ptychoX" / "__init__.py").exists():
        return None
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import ptychoX

    if Path(ptychoX.__file__).resolve().parent.parent != REF_DIR.resolve():
        raise RuntimeError(f"ptychoX imported from {ptychoX.__file__}, not from {REF_DIR}")
    return ptychoX


def host_threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:  # pragma: no cover - non-Linux
        return max(1, os.cpu_count() or 1)


def reference_sweep_fn(wl, ref, h, meas, scale, device="cpu", use_cuda_kernels=False):
    """One whole sweep through the reference's own PyTorch path, as its training drivers run it
    (``train_ptychography.py:549-557``, ``train_fpm.py:255-263``, ``train_coded.py:225-237``):
    the operator on complex64 tensors, ``F.mse_loss`` (or ``fd_loss``) against the observed
    amplitude ``sqrt(scale * counts)``, ``.backward()``.  Returns a callable giving the loss."""
    import torch
    import torch.nn.functional as F

    dev = torch.device(device)
    obj = torch.from_numpy(h["obj"]).to(dev).requires_grad_(True)
    aux = torch.from_numpy(h["aux"]).to(dev).requires_grad_(True)
    observed = torch.sqrt(torch.from_numpy(np.asarray(meas).astype(np.float32)).to(dev) * np.float32(scale))
    loss_fn = F.mse_loss
    if isinstance(wl, Coded):
        n = wl.n_obj
        t1 = (torch.ones((n, n), dtype=torch.complex64, device=dev) if h["t1"] is None
              else torch.from_numpy(h["t1"]).to(dev))
        t2 = torch.from_numpy(h["t2"]).to(dev)
        shifts = torch.from_numpy(np.asarray(h["pos"], dtype=np.float32)).to(dev)
        if wl.loss != "mse":
            from train_coded import fd_loss

            iso = wl.loss == "fd-isotropic"
            loss_fn = lambda a, b: fd_loss(a, b, isotropic=iso)  # noqa: E731

        def forward():
            return ref.ptychoX_coded(obj, aux, t1, t2, shifts, wl.ds, use_cuda_kernels=use_cuda_kernels)
    elif isinstance(wl, Fourier):
        led = torch.from_numpy(np.asarray(h["pos"], dtype=np.int64)).to(dev)

        def forward():
            return ref.ptychoX_fourier(obj, aux, led, use_cuda_kernels=use_cuda_kernels)
    elif isinstance(wl, ConventionalSubpixel):
        forward = reference_subpixel_forward(ref, obj, aux, h["pos"], use_cuda_kernels)
    else:
        pos = torch.from_numpy(np.asarray(h["pos"], dtype=np.int64)).to(dev)

        def forward():
            return ref.ptychoX_base(obj, aux, pos, use_cuda_kernels=use_cuda_kernels)

    def one():
        obj.grad = None
        aux.grad = None
        loss = loss_fn(forward(), observed)
        loss.backward()
        return loss.detach()

    return one


def reference_subpixel_forward(ref, obj, probe, positions, use_cuda_kernels=False):
    """The sub-pixel operator composed from the reference's own functions (it has none of its
    own): the window at floor(p + 1/2) cropped as base/ops.py:61-62 does, shifted by the
    fraction with shift_phase_ramp (coded/ops.py:157-171) on its spectrum, then ptychoX_base on
    the shifted patches.  Returns a callable giving the amplitudes."""
    import torch
    from ptychoX.coded.ops import shift_phase_ramp

    ph, pw = probe.shape
    pos = np.asarray(positions, dtype=np.float64)
    corner = np.floor(pos + 0.5)
    frac = pos - corner
    shifts = torch.from_numpy(np.stack([frac[:, 0] / pw, frac[:, 1] / ph], axis=1)).to(obj.device, obj.real.dtype)
    corners = corner.astype(np.int64).tolist()
    zero = torch.zeros(1, 2, dtype=torch.long, device=obj.device)

    def forward():
        ramp = shift_phase_ramp(ph, pw, shifts, obj.device, obj.real.dtype)
        crops = torch.stack([obj[y : y + ph, x : x + pw] for x, y in corners])
        patches = torch.fft.ifft2(torch.fft.fft2(crops) * ramp)
        return torch.cat([ref.ptychoX_base(patches[b], probe, zero, use_cuda_kernels=use_cuda_kernels)
                          for b in range(len(corners))], dim=0)

    return forward


def reference_counts(wl, ref, h, seed=7):
    """uint16 Poisson counts of the truth's forward model computed with the reference's own CPU
    operator (complex64), drawn by numpy; the workload's photon budget."""
    import torch

    from ptychox_b200 import synth

    t = torch.from_numpy
    with torch.no_grad():
        if isinstance(wl, Coded):
            n = wl.n_obj
            t1 = torch.ones((n, n), dtype=torch.complex64) if h["t1"] is None else t(h["t1"])
            amp = ref.ptychoX_coded(t(h["truth"]), t(h["aux"]), t1, t(h["t2"]),
                                    t(np.asarray(h["pos"], dtype=np.float32)), wl.ds)
        elif isinstance(wl, Fourier):
            amp = ref.ptychoX_fourier(t(h["truth"]), t(h["aux"]), t(np.asarray(h["pos"], dtype=np.int64)))
        elif isinstance(wl, ConventionalSubpixel):
            amp = reference_subpixel_forward(ref, t(h["truth"]), t(h["aux"]), h["pos"])()
        else:
            amp = ref.ptychoX_base(t(h["truth"]), t(h["aux"]), t(np.asarray(h["pos"], dtype=np.int64)))
    rng = np.random.default_rng(seed)
    return synth.poisson_counts(amp.numpy().astype(np.float64) ** 2, wl.photons, rng,
                                per_pixel=isinstance(wl, (Fourier, Coded)), brightest=isinstance(wl, Fourier))


def cpu_reference_rate(wl, host, measured, scale, budget_s: float = 12.0) -> dict | None:
    """Time the reference's own PyTorch CPU path (whole sweeps, all host threads) for about
    ``budget_s`` seconds after one warm-up sweep; None without the ``baseline/_ref`` install."""
    import torch

    ref = reference_package()
    if ref is None:
        return None
    threads = host_threads()
    prev = torch.get_num_threads()
    torch.set_num_threads(threads)
    try:
        one = reference_sweep_fn(wl, ref, host, measured, scale)
        t0 = time.perf_counter()
        one()
        first = time.perf_counter() - t0
        reps = int(max(1, min(10, budget_s / max(first, 1e-3))))
        t0 = time.perf_counter()
        for _ in range(reps):
            one()
        dt = (time.perf_counter() - t0) / reps
    finally:
        torch.set_num_threads(prev)
    return {"value": 1.0 / dt, "unit": "sweeps/s", "cores": threads, "kind": "reference",
            "sample": f"{reps} whole sweeps ({wl.batch} {wl.units} each) after one warm-up sweep; the reference's "
                      f"ptychoX (baseline/_ref) with use_cuda_kernels=False in complex64 + F.mse_loss (train_coded's fd_loss for the fd workloads) + backward, "
                      f"torch CPU on {threads} threads ({dt:.2f} s per sweep)"}


def reference_gpu_rates(wl, host, measured, scale, dev, flush, steps: int = 5, warmup: int = 2) -> dict | None:
    """The reference's own GPU paths on this B200, one request at a time: its PyTorch operator on
    CUDA tensors (torch.fft / cuFFT through ATen, ``use_cuda_kernels=False``) and its pybind11
    CUDA extension (``python/ptychoX/csrc``, built from source for sm_100a into baseline/_ref,
    ``use_cuda_kernels=True``), each a whole sweep per step (operator, F.mse_loss, backward)
    timed with CUDA events, L2 flushed between steps.  None without the reference install."""
    import importlib

    import torch

    ref = reference_package()
    if ref is None:
        return None
    out = {}
    for label, use_ext in (("torch_cuda", False), ("csrc_extension", True)):
        if use_ext and isinstance(wl, ConventionalSubpixel):
            continue
        try:
            one = reference_sweep_fn(wl, ref, host, measured, scale, device=dev, use_cuda_kernels=use_ext)
            for _ in range(warmup):
                one()
            torch.cuda.synchronize(dev)
            stream = torch.cuda.current_stream(dev)
            times = []
            for _ in range(steps):
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                one()
                b.record(stream)
                flush.zero_()
                torch.cuda.synchronize(dev)
                times.append(a.elapsed_time(b))
            ms = statistics.median(times)
            rec = {"value": 1e3 / ms, "unit": "sweeps/s", "ms_per_sweep": ms, "steps": steps}
            if use_ext:
                mod = {"Coded": "coded", "Fourier": "fpm"}.get(type(wl).__name__, "base")
                rec["module"] = str(Path(importlib.import_module(f"ptychoX.{mod}._C").__file__).relative_to(ROOT))
            out[label] = rec
        except Exception as e:  # report, do not fail the bench line
            out[label] = {"error": f"{type(e).__name__}: {e}"[:300]}
        torch.cuda.empty_cache()
    out["method"] = ("the reference's ptychoX (baseline/_ref), one whole sweep per step as its training drivers run "
                     "it: operator with use_cuda_kernels False (torch.fft on CUDA) or True (its cuFFT extension "
                     "compiled for sm_100a), F.mse_loss, backward; CUDA events, median of steps")
    return out


def cpu_sample_rate(wl, host, measured, scale, budget_s: float = 12.0) -> dict:
    """Time the CPU oracle (complex64, all host threads) on a bounded sample of the units."""
    from oracle import ptycho_oracle as O

    workers = O.default_workers()
    batch = wl.batch

    def run(k):
        t0 = time.perf_counter()
        wl.cpu_sweep(host, measured, scale, k, workers)
        return time.perf_counter() - t0

    k = min(batch, 4)
    run(k)  # warm-up (FFT plans, page faults)
    t = run(k)
    k2 = int(max(k, min(batch, budget_s / max(t / k, 1e-6))))
    t2 = run(k2)
    sweeps_per_s = (k2 / batch) / t2
    return {"value": sweeps_per_s, "unit": "sweeps/s", "cores": workers, "kind": "port",
            "sample": f"{k2} of {batch} {wl.units} per timed run, scaled to one sweep; complex64 numpy/scipy "
                      f"restatement of the reference torch CPU path ({t2:.1f} s)"}


# ---------------------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------------------


def run_reference(args) -> None:
    """The reference arm: the reference's own PyTorch CPU path on all host threads.

    Each step is one whole sweep (every position) of the workload through the unmodified
    ``ptychoX`` package of ``baseline/_ref`` (``use_cuda_kernels=False``, complex64,
    ``F.mse_loss`` + ``.backward()``), on the same seeded problem as our arm.  Without the
    install the oracle's numpy restatement runs instead, on a bounded sample of the units,
    and the line says ``kind: "port"``.  Under torchrun only rank 0 runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    wl = WORKLOADS[args.workload]
    h = wl.host(1000)
    batch = wl.batch
    ref = reference_package()
    threads = host_threads()
    if ref is not None:
        torch.set_num_threads(threads)
        meas, scale = reference_counts(wl, ref, h)
        h = dict(h)
        one = reference_sweep_fn(wl, ref, h, meas, scale)
        for _ in range(args.warmup):
            one()
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            one()
            times.append(time.perf_counter() - t0)
        per_sweep = statistics.mean(times)
        kind = "reference"
        sample = (f"whole sweeps ({batch} {wl.units} each): the reference's ptychoX from baseline/_ref, "
                  f"use_cuda_kernels=False, complex64, F.mse_loss (fd_loss for the fd workloads) + backward, "
                  f"torch CPU on {threads} threads")
    else:
        from oracle import ptycho_oracle as O

        workers = O.default_workers()
        rng = np.random.default_rng(7)

        def counts(k):
            if isinstance(wl, Coded):
                _, _, _, amp = O.coded_forward(h["truth"], h["aux"], h["t1"], h["t2"], h["pos"][:k], wl.ds,
                                               fp64=False, workers=workers)
            elif isinstance(wl, Fourier):
                amp, _, _ = O.fpm_forward(h["truth"], h["aux"], h["pos"][:k], fp64=False, workers=workers)
            elif isinstance(wl, ConventionalSubpixel):
                amp, _, _ = O.base_subpix_forward(h["truth"], h["aux"], h["pos"][:k], fp64=False, workers=workers)
            else:
                amp, _, _ = O.base_forward(h["truth"], h["aux"], h["pos"][:k], fp64=False, workers=workers)
            from ptychox_b200 import synth

            return synth.poisson_counts(amp.astype(np.float64) ** 2, wl.photons, rng,
                                        per_pixel=isinstance(wl, (Fourier, Coded)),
                                        brightest=isinstance(wl, Fourier))

        k = min(batch, 2)
        meas, scale = counts(k)
        wl.cpu_sweep(h, meas, scale, k, workers)
        t0 = time.perf_counter()
        wl.cpu_sweep(h, meas, scale, k, workers)
        per_unit = (time.perf_counter() - t0) / k
        n_units = int(min(batch, max(k, 2.0 / max(per_unit, 1e-6))))
        meas, scale = counts(n_units)
        for _ in range(args.warmup):
            wl.cpu_sweep(h, meas, scale, n_units, workers)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            wl.cpu_sweep(h, meas, scale, n_units, workers)
            times.append(time.perf_counter() - t0)
        per_sweep = statistics.mean(times) * batch / n_units
        kind = "port"
        threads = workers
        sample = (f"{n_units} of {batch} {wl.units} per step, scaled to one sweep; the oracle's complex64 "
                  "numpy/scipy restatement of the reference torch CPU path (baseline/_ref not installed)")
    value = 1.0 / per_sweep
    line = {
        "impl": "reference",
        "metric": wl.metric(),
        "value": value,
        "unit": "sweeps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per_sweep * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64",
        "data": "synthetic (seeded object and scan, Poisson uint16 counts from the forward model)",
        "config": wl.config(),
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# serving: the mixed stream (config 4)
# ---------------------------------------------------------------------------------------


def run_native(reqs, warm, dev, max_active):
    """The stream through the native server: each request submitted at its arrival time,
    all polled until finished; returns (results in rid order, wall seconds to the last)."""
    from ptychox_b200.native_server import NativeReconstructionServer

    with NativeReconstructionServer(dev.index or 0, max_active=max_active) as srv:
        srv.run(warm)
        pending = sorted(reqs, key=lambda r: (r.arrival, r.rid))
        ids, out = {}, {}
        t0 = time.perf_counter()
        while pending or ids:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                r = pending.pop(0)
                ids[srv.submit(r)] = r.rid
            for sid in list(ids):
                res = srv.poll(sid)
                if res is not None:
                    out[ids.pop(sid)] = res
            if ids or pending:
                time.sleep(5e-4)
        wall = time.perf_counter() - t0
    return [out[k] for k in sorted(out)], wall


def serving_record(args, dev) -> dict:
    """Served mixed stream vs one-at-a-time plain solves on the same GPU (config 4).

    The stream: ``--requests`` reconstructions (default 40), Poisson arrivals at 20/s,
    40/30/20/10 % from configs 0/2/3/1 with sizes jittered +-25 %, up to ``--iters`` (50)
    iterations each, stopping at a fixed error (``--target-ratio`` times the initial loss).
    Requests are synthesised (seeded, counts from the forward model) before the clock
    starts; their host arrays are uploaded at admission, inside the measured latency.  The
    same requests run through the Python server, the native server (``ptx_server_*``,
    submitted at their arrival times) and the plain loop (unfused operators,
    F.mse_loss, torch.optim.Adam, one request at a time)."""
    import torch

    from ptychox_b200 import _abi
    from ptychox_b200.serving import (ReconstructionServer, percentile, run_plain, serving_mix,
                                      synthesize_request)

    _abi.load()
    mix = serving_mix(args.requests, seed=4, rate=20.0)
    reqs = [synthesize_request(rid, m, t, size, seed=500 + rid, device=dev, iters=args.iters,
                               target_ratio=args.target_ratio)
            for rid, m, t, size in mix]
    torch.cuda.synchronize(dev)
    # warm-up: one small request of each modality and size class builds plans and loads kernels
    warm = [synthesize_request(1000 + i, m, 0.0, size, seed=900 + i, device=dev, iters=2)
            for i, (_, m, _, size) in enumerate({(m, size.get("p", size.get("n"))): (r, m, t, size)
                                                  for r, m, t, size in mix}.values())]
    ReconstructionServer(dev).run(warm, realtime=False)
    run_plain(warm, dev, realtime=False)

    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    launches0 = _abi.query("ptx_launch_count")
    t0 = time.perf_counter()
    served = ReconstructionServer(dev, max_active=args.max_active, units_per_cta=args.units_per_cta).run(
        reqs, realtime=True)
    t_served = time.perf_counter() - t0
    launches = _abi.query("ptx_launch_count") - launches0
    native, t_native = run_native(reqs, warm, dev, args.max_active)
    clk = clocks.stop()
    t0 = time.perf_counter()
    plain = run_plain(reqs, dev, realtime=True)
    t_plain = time.perf_counter() - t0

    def summary(results, wall):
        sweeps = sum(r.sweeps for r in results)
        lat = [r.latency for r in results]
        return {"wall_s": wall, "sweeps": sweeps, "sweeps_per_s": sweeps / wall, "p50_latency_s": percentile(lat, 50),
                "p99_latency_s": percentile(lat, 99), "iterations_mean": sweeps / max(len(results), 1)}

    def rel(a, b):
        return max(abs(x.final_loss - y.final_loss) / abs(y.final_loss) for x, y in zip(a, b))

    by_mod = {}
    for r in reqs:
        by_mod[r.modality] = by_mod.get(r.modality, 0) + 1
    sizes = sorted({(r.modality, tuple(r.aux0.shape)) for r in reqs})
    s_rate = sum(r.sweeps for r in served) / t_served
    n_rate = sum(r.sweeps for r in native) / t_native
    p_rate = sum(r.sweeps for r in plain) / t_plain
    return {
        "requests": len(reqs), "arrival_rate_per_s": 20.0, "max_active": args.max_active,
        "max_iterations_per_request": args.iters, "target_ratio": args.target_ratio, "mix": by_mod,
        "sizes": [f"{m} {'x'.join(map(str, sh))}" for m, sh in sizes],
        "mix_rule": "40/30/20/10% configs 0/2/3/1, sizes x U[0.75,1.25] (conventional probes {2,3,5}-smooth)",
        "served": summary(served, t_served),
        "native": summary(native, t_native),
        "plain": summary(plain, t_plain),
        "throughput_ratio_served_over_plain": s_rate / p_rate,
        "throughput_ratio_native_over_plain": n_rate / p_rate,
        "final_loss_rel_diff_max_served_vs_plain": rel(served, plain),
        "final_loss_rel_diff_max_native_vs_plain": rel(native, plain),
        "requests_stopped_at_target": {"served": sum(r.sweeps < args.iters for r in served),
                                       "native": sum(r.sweeps < args.iters for r in native),
                                       "plain": sum(r.sweeps < args.iters for r in plain)},
        # the servers keep up to two iterations of a request in flight, so a request that meets
        # its target may run one more before it is retired: its final loss is then lower
        "overshoot_iterations_mean_served_vs_plain": (sum(r.sweeps for r in served) - sum(r.sweeps for r in plain))
        / max(len(reqs), 1),
        "gpu_launches_served": launches,
        "clocks": clk,
        "methods": {"served": "Python server: HBM-budget admission, resident state, one captured graph per "
                              "reconstruction's iteration, concurrent replay on prioritised streams",
                    "native": "the same service in libptychox (ptx_server_*): scheduler thread replaying, "
                              "admission thread uploading / warming up / capturing / reading back; requests "
                              "submitted at their arrival times",
                    "plain": "one request at a time: unfused operators + F.mse_loss + torch.optim.Adam, the loss "
                             "read every iteration when a target is set (the reference drivers' loop)"},
    }


def run_serving(args) -> None:
    """The served mixed stream as its own bench line (``--workload serving-mix``)."""
    import torch

    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    rec = serving_record(args, dev)
    served = rec["served"]
    line = {
        "metric": "served mixed stream: sweeps/s (p50/p99 latency alongside)",
        "value": served["sweeps_per_s"],
        "unit": "sweeps/s",
        "n_gpus": 1,
        "steps": rec["requests"],
        "warmup": 0,
        "ms_per_step": 1e3 / max(served["sweeps_per_s"], 1e-9),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "c64 (FP32 FFT/constraint, FP64 loss sum)",
        "data": "synthetic (seeded problems, Poisson uint16 counts from the forward model)",
        "config": {"workload": "serving-mix", "requests": rec["requests"], "mix": rec["mix"]},
        "serving": rec,
        "gpu_launches": rec["gpu_launches_served"],
        "clocks": rec["clocks"],
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--scaling", default="strong", choices=["strong", "weak"],
                    help="N > 1: shard one reconstruction over the ranks (strong) or sweep all units on every rank")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS) + ["serving-mix"])
    ap.add_argument("--requests", type=int, default=40)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--target-ratio", type=float, default=0.25,
                    help="serving: stop a request once its loss is at most this fraction of its initial loss "
                         "(0: run every request for --iters iterations)")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the served-stream record of the default line")
    ap.add_argument("--max-active", type=int, default=8)
    ap.add_argument("--units-per-cta", type=int, default=8,
                    help="serving: bound on the units a persistent-pass CTA takes (0: one wave)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU paths (torch on CUDA, its CUDA extension)")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--units", type=int, default=0,
                    help="run the workload on its first N scan units only (small profiling cases)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "serving-mix":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the served stream has no CPU reference arm; "
                              "its plain baseline is timed in the same run"}), flush=True)
            return
        run_serving(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
