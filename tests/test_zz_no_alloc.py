"""The allocation-free sweep entry point against the workspace one, through the C ABI.

ptx_base_sweep_noalloc exists for callers that cannot allocate device memory (plug-in
hosts that keep the GPU memory pool to themselves, acquisition loops that must not take
a cudaMalloc's synchronisation); its scratch is a fixed 8 MiB device array inside the
library.  This file is collected last so a failure here leaves every other test run.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _problem():
    from ptychox_b200 import synth

    rng = np.random.default_rng(77)
    obj = synth.random_object(640, 640, rng)
    probe = synth.gaussian_probe(256, 256, rng)
    pos = synth.raster_positions(6, 60, 10, 3, rng)  # 36 positions: chunks of 15, 15 and 6 frames
    meas = rng.poisson(30.0, size=(len(pos), 256, 256)).astype(np.uint16)
    guess = (obj * (1 + 0.1 * rng.standard_normal(obj.shape))).astype(np.complex64)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return t(guess), t(probe), t(pos), t(meas), 0.01


def _noalloc(lib, s, p, pos, meas, scale):
    loss = torch.empty((), dtype=torch.float64, device="cuda")
    gs = torch.empty_like(s)
    gp = torch.empty_like(p)
    st = lib.ptx_base_sweep_noalloc(s.data_ptr(), s.shape[0], s.shape[1], p.data_ptr(), p.shape[0], p.shape[1],
                                    pos.data_ptr(), pos.shape[0], meas.data_ptr(), C.c_float(scale),
                                    loss.data_ptr(), gs.data_ptr(), gp.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.ptx_last_error()
    torch.cuda.synchronize()
    return float(loss.item()), gs.cpu().numpy(), gp.cpu().numpy()


# PTX_NOALLOC_SCRATCH_BYTES of include/ptychox.h and the workspace header (error word and the
# 65536-entry float count-decode table)
NOALLOC_SCRATCH_BYTES = 8 * 1024 * 1024
HEADER_BYTES = 256 + 65536 * 4


def test_noalloc_matches_workspace_sweep_twice():
    """Two calls in a row against the one-chunk workspace sweep and the FP64 oracle.  The
    shared array holds fewer frames than the scan, so the no-alloc call runs several chunks
    (reusing the array within the call) while the reference call runs one."""
    from oracle import ptycho_oracle as O
    from ptychox_b200 import _abi
    from ptychox_b200.base import base_sweep

    lib = _abi.load()
    s, p, pos, meas, scale = _problem()
    frame_bytes = p.shape[0] * p.shape[1] * 8
    assert (NOALLOC_SCRATCH_BYTES - HEADER_BYTES) // frame_bytes < pos.shape[0]
    assert lib.ptx_base_workspace_bytes(p.shape[0], p.shape[1], pos.shape[0]) >= HEADER_BYTES + pos.shape[0] * frame_bytes
    rl, rs, rp = O.base_sweep(s.cpu().numpy(), p.cpu().numpy(), pos.cpu().numpy(), meas.cpu().numpy(), scale)
    ref_loss, ref_gs, ref_gp = base_sweep(s, p, pos, meas, scale)
    ref_loss = float(ref_loss.item())
    ref_gs, ref_gp = ref_gs.cpu().numpy(), ref_gp.cpu().numpy()
    assert abs(ref_loss - rl) <= TOL * abs(rl)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        loss, gs, gp = _noalloc(lib, s, p, pos, meas, scale)
        assert abs(loss - ref_loss) <= TOL * abs(ref_loss)
        assert rel_l2(gs, ref_gs) < TOL
        assert rel_l2(gp, ref_gp) < TOL
        assert abs(loss - rl) <= TOL * abs(rl)
        assert rel_l2(gs, rs) < TOL
        assert rel_l2(gp, rp) < TOL


def test_noalloc_rejects_frames_beyond_its_scratch():
    from ptychox_b200 import _abi

    lib = _abi.load()
    s = torch.zeros(1024, 1024, dtype=torch.complex64, device="cuda")
    p = torch.zeros(1024, 1024, dtype=torch.complex64, device="cuda")
    pos = torch.zeros(1, 2, dtype=torch.long, device="cuda")
    meas = torch.zeros(1, 1024, 1024, dtype=torch.int32, device="cuda").to(torch.uint16)
    out = torch.empty((), dtype=torch.float64, device="cuda")
    st = lib.ptx_base_sweep_noalloc(s.data_ptr(), 1024, 1024, p.data_ptr(), 1024, 1024, pos.data_ptr(), 1,
                                    meas.data_ptr(), C.c_float(1.0), out.data_ptr(), s.data_ptr(), p.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    assert st == _abi.PTX_ERR_WORKSPACE
    assert "scratch" in lib.ptx_last_error().decode()
