"""Data-parallel sweep logic on two gloo ranks (CPU): sharded oracle sweeps reduced with
``reduce_sweep`` equal the single-process sweep over all positions."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT, rel_l2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(kind):
    import sys

    sys.path.insert(0, str(ROOT))
    from oracle import ptycho_oracle as O
    from ptychox_b200 import synth

    rng = np.random.default_rng(21)
    if kind == "base-config0":
        # config 0 shape: 512^2 object, 128^2 probe, 11 x 11 raster step 32, U[-2, 2] jitter
        obj = synth.random_object(512, 512, rng)
        probe = synth.gaussian_probe(128, 128, rng)
        pos = synth.raster_positions(11, 32, 8, 2, rng)
        amp, _, _ = O.base_forward(obj, probe, pos)
        meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
        return obj, probe, pos, meas, scale
    if kind == "base":
        obj = synth.random_object(96, 96, rng)
        probe = synth.gaussian_probe(32, 32, rng)
        pos = synth.raster_positions(5, 14, 2, 2, rng)
        amp, _, _ = O.base_forward(obj, probe, pos)
        meas, scale = synth.poisson_counts(amp**2, 1e4, rng)
        return obj, probe, pos, meas, scale
    obj = synth.random_object(64, 64, rng)
    pupil = synth.circular_pupil(16, 0.3)
    led = np.array([[24 + dx, 24 + dy] for dy in (-8, 0, 8) for dx in (-8, 0, 8)], np.int64)
    amp, _, _ = O.fpm_forward(obj, pupil, led)
    meas, scale = synth.poisson_counts(amp**2, 300.0, rng, per_pixel=True)
    return obj, pupil, led, meas, scale


def _worker(rank, world, port, kind, out):
    import sys

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from oracle import ptycho_oracle as O
    from ptychox_b200.distributed import reduce_sweep, shard_positions

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        obj, aux, pos, meas, scale = _problem(kind)
        idx = shard_positions(pos, rank, world)
        sweep = O.fpm_sweep if kind == "fpm" else O.base_sweep
        loss, g1, g2 = sweep(obj, aux, pos[idx], meas[idx], scale)
        t_loss = torch.tensor(loss, dtype=torch.float64)
        t1 = torch.from_numpy(np.ascontiguousarray(g1))
        t2 = torch.from_numpy(np.ascontiguousarray(g2))
        reduce_sweep(t_loss, [t1, t2], len(idx), len(pos))
        if rank == 0:
            out.put((float(t_loss), t1.numpy(), t2.numpy(), [len(shard_positions(pos, r, world)) for r in range(world)]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["base", "fpm", "base-config0"])
def test_two_rank_sweep_equals_single_process(kind):
    """One reconstruction sharded over two ranks (row bands, uneven: 13 / 12, and 61 / 60 at the
    config-0 shape) and reduced with reduce_sweep equals the single-process sweep."""
    from oracle import ptycho_oracle as O

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    loss, g1, g2, sizes = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    obj, aux, pos, meas, scale = _problem(kind)
    sweep = O.fpm_sweep if kind == "fpm" else O.base_sweep
    rl, r1, r2 = sweep(obj, aux, pos, meas, scale)
    assert sum(sizes) == len(pos) and max(sizes) - min(sizes) <= 1
    assert abs(loss - rl) <= 1e-12 * abs(rl)
    assert rel_l2(g1, r1) < 1e-12
    assert rel_l2(g2, r2) < 1e-12


def test_shards_are_row_bands():
    from ptychox_b200.distributed import shard_positions

    rng = np.random.default_rng(0)
    pos = rng.integers(0, 1000, size=(101, 2))
    parts = [shard_positions(pos, r, 4) for r in range(4)]
    assert sorted(np.concatenate(parts).tolist()) == list(range(101))
    ys = [pos[p, 1] for p in parts]
    for a, b in zip(ys, ys[1:]):
        assert a.max() <= b.min()
    with pytest.raises(ValueError):
        shard_positions(pos, 4, 4)
