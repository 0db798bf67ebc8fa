"""Gradient harness over the discrete adjoint: a torch.autograd.Function whose forward
runs nsteps FP64 time steps through the C ABI (awfl_step) with a checkpoint every
``ckpt_every`` steps, and whose backward calls awfl_step_adjoint once per segment, last
segment first. The time step dt is a fixed parameter (no gradient).

    ctx = capi.Context(32, 32, 16)
    s0 = ctx.new_state(); ctx.init_state(s0, kind=capi.INIT_BUBBLE)
    s0.requires_grad_(True)
    sN = euler_steps(s0, ctx, nsteps=20, dt=dt, ckpt_every=10)
    J = 0.5 * ((sN[4] - target) ** 2).sum()
    J.backward()          # s0.grad = dJ/dS0 (halo entries zero)

Halo entries of the result are recomputed from the interior by every step, so they carry
no gradient; s0.grad is zero there.
"""
from __future__ import annotations

import torch


class EulerSteps(torch.autograd.Function):
    @staticmethod
    def forward(fctx, state0, context, nsteps, dt, ckpt_every):
        if nsteps < 0 or ckpt_every < 1:
            raise ValueError("nsteps must be >= 0 and ckpt_every >= 1")
        s = state0.detach().clone()
        ckpts = []
        for n in range(nsteps):
            if n % ckpt_every == 0:
                ckpts.append((s.clone(), context.dimswitch))
            context.step(s, dt)
        fctx.context, fctx.dt, fctx.nsteps, fctx.every = context, dt, nsteps, ckpt_every
        fctx.ckpts = ckpts
        fctx.final_dimswitch = context.dimswitch
        return s

    @staticmethod
    def backward(fctx, grad_out):
        context, dt, nsteps, every = fctx.context, fctx.dt, fctx.nsteps, fctx.every
        lam = grad_out.detach().contiguous().clone()
        for seg in range(len(fctx.ckpts) - 1, -1, -1):
            ckpt, ds = fctx.ckpts[seg]
            n = min(every, nsteps - seg * every)
            context.dimswitch = ds
            context.step_adjoint(ckpt, lam, n, dt)
        context.dimswitch = fctx.final_dimswitch
        return lam, None, None, None, None


def euler_steps(state0, context, nsteps, dt, ckpt_every=20):
    """nsteps time steps of ``context`` (an FP64 capi.Context) from state0, differentiable
    with respect to state0."""
    return EulerSteps.apply(state0, context, int(nsteps), float(dt), int(ckpt_every))
