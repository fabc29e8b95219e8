"""torch.autograd binding of the FDTD adjoint (used only for optimisation).

    ir = ReceiverIR.apply(coef, signal, sim, steps, every)

coef   [M][S][5] boundary filter coefficients {b0 b1 b2 a1 a2} (any float
       dtype, CPU); the forward pass runs with them rounded to float32
signal [n_src][steps] source signals (float32, CPU)
sim    a classified capi.Simulation with sources and receivers set
returns the receiver samples [n_rcv][steps] (float32, CPU).

The forward pass is virs_forward_checkpointed (checkpoints every `every`
steps); the backward pass is virs_adjoint, which recomputes each segment
once and runs the step backwards in time on the GPU.  Gradients are with
respect to the float32 coefficients the kernel uses (FP64 accumulation).
"""
from __future__ import annotations

import numpy as np
import torch

from . import capi


class ReceiverIR(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coef: torch.Tensor, signal: torch.Tensor, sim: "capi.Simulation", steps: int, every: int = 64):
        c = coef.detach().to(torch.float32).cpu().numpy()
        M, S, _ = c.shape
        sim.set_filters(c, n_sections=S)
        src = sim._src_idx
        sim.set_sources(src, signal.detach().to(torch.float32).cpu().numpy())
        sim.set_receivers(sim._rcv_idx)
        sim.forward_checkpointed(steps, every)
        ir = torch.from_numpy(sim.ir(0, steps).copy())
        ctx.sim, ctx.shape = sim, (M, S)
        ctx.coef_dtype = coef.dtype
        return ir

    @staticmethod
    def backward(ctx, grad_ir: torch.Tensor):
        M, S = ctx.shape
        gc, gs = ctx.sim.adjoint(grad_ir.detach().to(torch.float32).cpu().numpy(), M, S)
        return (torch.from_numpy(gc).to(ctx.coef_dtype), torch.from_numpy(np.ascontiguousarray(gs)), None, None, None)


def attach(sim: "capi.Simulation", src_idx, rcv_idx) -> "capi.Simulation":
    """Remember the source and receiver voxels the autograd function re-applies."""
    sim._src_idx = np.asarray(src_idx, np.uint64)
    sim._rcv_idx = np.asarray(rcv_idx, np.uint64)
    return sim
