"""Fused Adam for complex parameters with resident state (one library call per step).

Semantics of ``torch.optim.Adam`` on complex tensors (the reference drivers' optimiser,
``train_ptychography.py:500-507``: betas (0.9, 0.999), eps 1e-16) plus the drivers'
optional projections.  The state (moments and the step count) lives on the device, so a
step can be captured in a CUDA graph and replayed.
"""

from __future__ import annotations

import torch

from . import _abi
from ._utils import ptr, stream_handle

__all__ = ["FusedAdam", "CONSTRAINTS"]

CONSTRAINTS = {
    None: _abi.PTX_CONSTRAIN_NONE,
    "none": _abi.PTX_CONSTRAIN_NONE,
    "unit_amplitude": _abi.PTX_CONSTRAIN_UNIT_AMPLITUDE,
    "real_nonnegative": _abi.PTX_CONSTRAIN_REAL_NONNEGATIVE,
}


class FusedAdam:
    """Adam over complex64 CUDA parameters; ``step(grads)`` updates them in place."""

    def __init__(self, params, lrs, betas=(0.9, 0.999), eps=1e-16, constraints=None):
        self.params = list(params)
        if isinstance(lrs, (int, float)):
            lrs = [float(lrs)] * len(self.params)
        self.lrs = [float(x) for x in lrs]
        self.betas = (float(betas[0]), float(betas[1]))
        self.eps = float(eps)
        cons = constraints if constraints is not None else [None] * len(self.params)
        self.constraints = [CONSTRAINTS[c] for c in cons]
        for p in self.params:
            if not (p.is_cuda and p.dtype == torch.complex64 and p.is_contiguous()):
                raise TypeError("FusedAdam parameters must be contiguous complex64 CUDA tensors")
        self.exp_avg = [torch.zeros_like(p) for p in self.params]
        self.exp_avg_sq = [torch.zeros_like(p) for p in self.params]
        self.state = [torch.zeros(4, dtype=torch.int32, device=p.device) for p in self.params]

    @torch.no_grad()
    def step(self, grads) -> None:
        for p, g, m, v, st, lr, c in zip(self.params, grads, self.exp_avg, self.exp_avg_sq, self.state, self.lrs,
                                          self.constraints):
            g = g.contiguous()
            _abi.call("ptx_adam_step", ptr(p), ptr(g), ptr(m), ptr(v), p.numel(), ptr(st), lr, self.betas[0],
                      self.betas[1], self.eps, c, stream_handle(p.device))

    @property
    def step_count(self) -> int:
        return int(self.state[0][0].item())
