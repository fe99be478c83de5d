"""Fused Adam step vs torch.optim.Adam (FP32, the reference drivers' optimiser) and the oracle."""

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import ptycho_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 4096, 100003])
def test_matches_torch_adam(n):
    from ptychox_b200.optim import FusedAdam

    rng = np.random.default_rng(n)
    p0 = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    p_ref = torch.from_numpy(p0.copy()).cuda().requires_grad_(True)
    ref = torch.optim.Adam([p_ref], lr=0.01, betas=(0.9, 0.999), eps=1e-16)
    p = torch.from_numpy(p0.copy()).cuda()
    fused = FusedAdam([p], [0.01])
    po, mo, vo = p0.copy(), np.zeros_like(p0), np.zeros_like(p0)
    for step in range(1, 6):
        g = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64) * (0.1 * step)
        p_ref.grad = torch.from_numpy(g).cuda()
        ref.step()
        fused.step([torch.from_numpy(g).cuda()])
        po, mo, vo = O.adam_step(po, g, mo, vo, step, 0.01)
    assert fused.step_count == 5
    assert rel_l2(p.cpu().numpy(), p_ref.detach().cpu().numpy()) < 1e-6
    assert rel_l2(p.cpu().numpy(), po) < 1e-6


def test_constraints_and_graph_replay():
    from ptychox_b200.optim import FusedAdam

    rng = np.random.default_rng(1)
    p0 = (2 * rng.standard_normal(1000) + 2j * rng.standard_normal(1000)).astype(np.complex64)
    a = torch.from_numpy(p0.copy()).cuda()
    b = torch.from_numpy(p0.copy()).cuda()
    opt = FusedAdam([a, b], [0.05, 0.05], constraints=["unit_amplitude", "real_nonnegative"])
    g = torch.from_numpy((rng.standard_normal(1000) + 1j * rng.standard_normal(1000)).astype(np.complex64)).cuda()
    # capture one step in a CUDA graph and replay it: the device step counter advances
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        graph.capture_begin(capture_error_mode="relaxed")
        opt.step([g, g])
        graph.capture_end()
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    assert opt.step_count == 3
    pa, pb = a.cpu().numpy(), b.cpu().numpy()
    assert np.abs(pa).max() <= 1.0 + 1e-6
    assert (pb.imag == 0).all() and (pb.real >= 0).all()
    ra, rb = p0.copy(), p0.copy()
    ma, va, mb, vb = (np.zeros_like(p0) for _ in range(4))
    gn = g.cpu().numpy()
    for step in range(1, 4):
        ra, ma, va = O.adam_step(ra, gn, ma, va, step, 0.05, constraint="unit_amplitude")
        rb, mb, vb = O.adam_step(rb, gn, mb, vb, step, 0.05, constraint="real_nonnegative")
    assert rel_l2(pa, ra) < 1e-6 and rel_l2(pb, rb) < 1e-6
