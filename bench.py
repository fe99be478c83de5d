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
``--impl reference`` times the reference algorithm's CPU restatement (the oracle) on
all host cores on a bounded sample of the same workload.

With N > 1 (torchrun) each rank sweeps its own 900 positions over the shared object
and the gradients are all-reduced over NCCL (data-parallel sweep, weak scaling).
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

WORKLOADS = {
    # name: (object side, probe side, raster grid, step, origin, jitter, photons)
    "conventional-900x512-2048": (2048, 512, 30, 48, 64, 3, 1e5),
    "conventional-121x128-512": (512, 128, 11, 32, 8, 2, 1e4),
}
DEFAULT_WORKLOAD = "conventional-900x512-2048"


def conventional_bytes_model(n_obj: int, p: int, batch: int) -> float:
    """Algorithmic HBM bytes of one conventional sweep.

    Per position: 8 P^2 (object window gather) + 2 P^2 (uint16 counts) + 16 P^2
    (object-gradient read-modify-write); per sweep: + 16 P^2 (probe in, probe gradient
    out) + 8 N^2 (zeroing the object gradient).
    """
    p2 = float(p) * p
    return 26.0 * p2 * batch + 16.0 * p2 + 8.0 * float(n_obj) ** 2


def hbm_peak() -> tuple[float, str]:
    try:
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def synth_conventional(name: str, seed: int, device):
    """Seeded cfg inputs: truth -> CUDA forward -> Poisson counts; evaluation point = perturbed truth."""
    import torch

    from ptychox_b200 import ptychoX_base, synth

    n_obj, p, grid, step, origin, jitter, photons = WORKLOADS[name]
    rng = np.random.default_rng(seed)
    obj_true = synth.random_object(n_obj, n_obj, rng)
    probe = synth.gaussian_probe(p, p, rng)
    pos = synth.raster_positions(grid, step, origin, jitter, rng)
    s = torch.from_numpy(obj_true).to(device)
    pr = torch.from_numpy(probe).to(device)
    pd = torch.from_numpy(pos).to(device)
    with torch.no_grad():
        amp = ptychoX_base(s, pr, pd)
        inten = amp.double() ** 2
        scale = float(np.float32(float(inten.sum(dim=(1, 2)).mean()) / photons))
        gen = torch.Generator(device=device).manual_seed(seed)
        counts = torch.poisson(inten / scale, generator=gen)
        if float(counts.max()) > 65535:
            raise RuntimeError("synthetic counts saturate uint16")
        meas = counts.to(torch.int32).to(torch.uint16)
        del amp, inten, counts
    guess = (obj_true * (1 + 0.1 * rng.standard_normal(obj_true.shape))).astype(np.complex64)
    return {
        "sample": torch.from_numpy(guess).to(device),
        "probe": pr,
        "positions": pd,
        "measured": meas,
        "scale": scale,
        "host": {"sample": guess, "probe": probe, "positions": pos},
        "n_obj": n_obj,
        "p": p,
        "batch": len(pos),
    }


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


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from ptychox_b200 import _abi, ptychoX_base_loss
    from ptychox_b200.base import base_sweep
    from ptychox_b200._utils import workspace

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    _abi.load()

    prob = synth_conventional(args.workload, seed=1000 + rank, device=dev)
    s, pr, pos, meas, scale = prob["sample"], prob["probe"], prob["positions"], prob["measured"], prob["scale"]
    ph = pw = prob["p"]
    batch = prob["batch"]
    ws = workspace(_abi.query("ptx_base_workspace_bytes", ph, pw, batch), dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        loss, gs, gp = base_sweep(s, pr, pos, meas, scale, ws=ws)
        if world > 1:
            dist.all_reduce(gs)
            dist.all_reduce(gp)
            dist.all_reduce(loss)
        return loss

    def timed(k: int, fn) -> list[float]:
        times = []
        stream = torch.cuda.current_stream(dev)
        for _ in range(k):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            flush.zero_()  # write > L2 between timed steps (outside the events)
            times.append((a, b))
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in times]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    # ---- timed region -------------------------------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
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
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms / 1e3)

    # ---- roofline: the sweep's kernels timed with library events ------------------
    _abi.query("ptx_profile_reset")
    _abi.query("ptx_profile_enable", 1)
    prof_ms = timed(args.steps, step)
    _abi.query("ptx_profile_enable", 0)
    per_kernel = _abi.profile_read()
    sweep_bytes = conventional_bytes_model(prob["n_obj"], ph, batch)
    peak, peak_kind = hbm_peak()
    sweep_ms = statistics.median(prof_ms)
    achieved = sweep_bytes / (ms_per_step / 1e3) / 1e9
    kernels = []
    kern_total = sum(v[0] for v in per_kernel.values()) or 1.0
    for name, (ms, n) in sorted(per_kernel.items(), key=lambda kv: -kv[1][0]):
        kernels.append({"name": name, "launches_per_step": n / args.steps, "ms_per_launch": ms / n,
                        "share": ms / kern_total})
    roofline = {
        "bound": "hbm",
        "achieved": achieved,
        "peak": peak,
        "unit": "GB/s",
        "frac": achieved / peak,
        "traffic": None,
        "peak_kind": f"{peak_kind} hbm_gbs",
        "scope": "fused sweep (all passes of one sweep, CUDA events on its stream)",
        "algorithmic_bytes_per_sweep": sweep_bytes,
        "profiled_sweep_ms": sweep_ms,
        "kernels": kernels,
    }

    # ---- e2e: public API with pinned host buffers -----------------------------------
    host = prob["host"]
    hs = torch.from_numpy(host["sample"]).pin_memory()
    hp = torch.from_numpy(host["probe"]).pin_memory()
    hpos = torch.from_numpy(host["positions"]).pin_memory()
    out_gs = torch.empty_like(hs).pin_memory()
    out_gp = torch.empty_like(hp).pin_memory()
    out_loss = torch.empty((), dtype=torch.float64).pin_memory()

    def e2e_step():
        ds = hs.to(dev, non_blocking=True).requires_grad_(True)
        dp = hp.to(dev, non_blocking=True).requires_grad_(True)
        dpos = hpos.to(dev, non_blocking=True)
        loss = ptychoX_base_loss(ds, dp, dpos, meas, scale)
        loss.backward()
        if world > 1:
            dist.all_reduce(ds.grad)
            dist.all_reduce(dp.grad)
        out_gs.copy_(ds.grad, non_blocking=True)
        out_gp.copy_(dp.grad, non_blocking=True)
        out_loss.copy_(loss.detach(), non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    e2e_ms = sum(timed(args.steps, e2e_step))
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = hs.numel() * 8 + hp.numel() * 8 + hpos.numel() * 8
    d2h = out_gs.numel() * 8 + out_gp.numel() * 8 + 8
    e2e = {"value": world * args.steps / (e2e_ms / 1e3), "unit": "sweeps/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h,
           "note": "measured counts resident in HBM (uploaded once, as in the reference training loop); "
                   "object, probe, positions uploaded and loss + gradients read back every step"}

    # ---- CPU baseline (rank 0, N = 1) --------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample_rate(host, meas.cpu().numpy(), scale, budget_s=args.cpu_budget)

    if rank == 0:
        n_obj, p = prob["n_obj"], ph
        line = {
            "metric": f"fwd+adj sweeps/s ({batch}×{p}²→{n_obj}²)",
            "value": value,
            "unit": "sweeps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "c64 (FP32 FFT/constraint, FP64 loss sum)",
            "data": "synthetic (seeded object/probe/raster, Poisson uint16 counts)",
            "config": {
                "workload": args.workload,
                "positions": batch,
                "probe": [p, p],
                "object": [n_obj, n_obj],
                "parallelism": f"dp{world}" if world > 1 else "single GPU",
                "l2": "flushed between timed steps (256 MB write outside the step events)",
            },
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def cpu_sample_rate(host, measured, scale, budget_s: float = 12.0) -> dict:
    """Time the CPU oracle (complex64, all host threads) on a bounded sample of positions."""
    from oracle import ptycho_oracle as O

    workers = O.default_workers()
    pos = host["positions"]
    batch = len(pos)

    def run(k):
        t0 = time.perf_counter()
        O.base_sweep(host["sample"], host["probe"], pos[:k], measured[:k], scale, fp64=False, workers=workers)
        return time.perf_counter() - t0

    k = min(batch, 16)
    t = run(k)
    per_pos = t / k
    k2 = int(max(k, min(batch, budget_s / max(per_pos, 1e-6))))
    t2 = run(k2)
    sweeps_per_s = (k2 / batch) / t2
    return {"value": sweeps_per_s, "unit": "sweeps/s", "cores": workers, "kind": "port",
            "sample": f"{k2} of {batch} positions per timed run, scaled to one sweep; complex64 numpy/scipy "
                      f"restatement of the reference torch CPU path ({t2:.1f} s)"}


# ---------------------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------------------


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ptycho_oracle as O
    from ptychox_b200 import synth

    n_obj, p, grid, step_px, origin, jitter, photons = WORKLOADS[args.workload]
    rng = np.random.default_rng(1000)
    obj = synth.random_object(n_obj, n_obj, rng)
    probe = synth.gaussian_probe(p, p, rng)
    pos = synth.raster_positions(grid, step_px, origin, jitter, rng)
    batch = len(pos)
    workers = O.default_workers()
    # a bounded sample per step: enough positions for ~2 s of work
    k = min(batch, 8)
    amp, _, _ = O.base_forward(obj, probe, pos[:k], fp64=False, workers=workers)
    t0 = time.perf_counter()
    O.base_forward(obj, probe, pos[:k], fp64=False, workers=workers)
    per_pos = (time.perf_counter() - t0) / k * 3.0
    sample = int(min(batch, max(k, 2.0 / max(per_pos, 1e-6))))
    amp, _, _ = O.base_forward(obj, probe, pos[:sample], fp64=False, workers=workers)
    meas, scale = synth.poisson_counts(amp.astype(np.float64) ** 2, photons, rng)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)

    def one():
        O.base_sweep(guess, probe, pos[:sample], meas, scale, fp64=False, workers=workers)

    for _ in range(args.warmup):
        one()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
    per_sweep = statistics.mean(times) * batch / sample
    value = 1.0 / per_sweep
    line = {
        "impl": "reference",
        "metric": f"fwd+adj sweeps/s ({batch}×{p}²→{n_obj}²)",
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
        "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "positions": batch, "probe": [p, p], "object": [n_obj, n_obj]},
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": workers, "kind": "port",
                         "sample": f"{sample} of {batch} positions per step, scaled to one sweep"},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
