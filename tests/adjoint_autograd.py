"""Test-harness wrapper of the discrete adjoint as a torch.autograd.Function.

RK3Frozen.apply(U0, solver, dt, nsteps, ckpt_every) returns U^N of nsteps
frozen-dt SSP-RK3 steps run by cfd_adjoint_record; its backward is
cfd_adjoint_reverse. Tensors are host (CPU) float64 tensors in the reference's
AoS layout [ncell, nvar], as the C ABI takes them; torch only carries the
gradient bookkeeping here.
"""
from __future__ import annotations

import numpy as np
import torch


class RK3Frozen(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, solver, dt, nsteps, ckpt_every):
        solver.set_cons(U0.detach().cpu().numpy())
        solver.adjoint_record(float(dt), int(nsteps), int(ckpt_every))
        ctx.solver = solver
        return torch.from_numpy(np.ascontiguousarray(solver.cons))

    @staticmethod
    def backward(ctx, grad_UN):
        g = ctx.solver.adjoint_reverse(np.ascontiguousarray(grad_UN.detach().cpu().numpy(), dtype=np.float64))
        return torch.from_numpy(g), None, None, None, None
