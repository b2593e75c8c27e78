"""Differentiable inverse-KS loss: torch.autograd.Function over the C ABI.

forward:  v_xc (float64 tensor on the child nodes) -> eigensolve -> rho -> L
          (invdft_solve_eigen; the eigenvectors stay on the GPU, stored once)
backward: the hand-written adjoint -- block MINRES for every state plus the
          projection of psi_i p_i onto the v_xc nodes (invdft_force_backward)
          -- returns dL/dv_xc; no Krylov vectors are kept after it returns.

L is the reference's loss sum_q w (rho*_up - rho/2)^2 JxW
(InverseDFTSolverFunction.cpp:893-900); with unit weights this is
(1/4) int (rho - rho*)^2.  Its gradient is the reference's force vector, whose
constrained (hanging) entries are zero.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .native import Stats, f64, ptr
from .solver import InverseDFTSolverFunction, _check


class InverseKSLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vxc: torch.Tensor, fn: InverseDFTSolverFunction):
        pot = f64(vxc.detach().cpu().numpy()).copy()
        st = Stats()
        _check(fn.lib, fn.ctx, fn.lib.invdft_solve_eigen(fn.ctx, ptr(pot), C.byref(st)))
        ctx.fn = fn
        ctx.generation = int(st.generation)
        ctx.device, ctx.dtype = vxc.device, vxc.dtype
        fn.last_stats = st.as_dict()
        return torch.tensor(st.loss, dtype=torch.float64, device=vxc.device)

    @staticmethod
    def backward(ctx, grad_L):
        fn = ctx.fn
        force = np.zeros(fn.n_child)
        st = Stats()
        # the library refuses (NOT_READY) if any forward evaluation or potential
        # change ran on this context after this forward
        _check(fn.lib, fn.ctx, fn.lib.invdft_force_backward_at(fn.ctx, ctx.generation, ptr(force), C.byref(st)))
        fn.last_backward_stats = st.as_dict()
        g = torch.from_numpy(force).to(device=ctx.device, dtype=ctx.dtype)
        return grad_L * g, None


def inverse_ks_loss(vxc: torch.Tensor, fn: InverseDFTSolverFunction) -> torch.Tensor:
    """L(v_xc) with an adjoint-based gradient."""
    return InverseKSLoss.apply(vxc, fn)
