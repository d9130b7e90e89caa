"""Reverse-mode differentiation of a rollout of hydro steps behind ``torch.autograd.Function``.

The forward runs ``steps`` static-mesh steps (``time_step`` + ``step``) on the GPU through the C ABI and keeps a
checkpoint of Q every ``every`` steps plus the dt of every step. The backward walks the segments from the last to the
first: it restores the segment's checkpoint, recomputes the segment's states forward, and runs the hand-written adjoint
kernels (``luna_fv_step_adjoint``: Qbar^n = J^T Qbar^n+1 at fixed dt) from the segment's last step to its first. Memory:
one checkpoint per segment plus the states of one segment, instead of every state of the rollout; cost: one extra forward
of each step. The dt of each step is held fixed in the derivative (the reference's step_adjoint does the same,
finite_volume.hpp:2196-2231); pass ``dts`` to replay a given schedule (finite differences of the same map).
"""
from __future__ import annotations

import torch

from . import hydro


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0, fv, steps, courant=0.3, every=20, dts=None):
        if not (q0.is_cuda and q0.dtype == torch.float64):
            raise ValueError("q0 must be a CUDA float64 tensor [N, D + 2]")
        q = q0.detach().contiguous().clone()
        fv.set_state(q)
        checkpoints = {}
        used = []
        for s in range(steps):
            if s % every == 0:
                checkpoints[s] = fv.get_state(torch.empty_like(q))
            dt = fv.time_step(courant)
            if dts is not None:
                dt = float(dts[s])
            fv.step(dt)
            used.append(dt)
        out = fv.get_state(torch.empty_like(q))
        ctx.fv, ctx.steps, ctx.courant, ctx.every = fv, steps, courant, every
        ctx.checkpoints, ctx.dts = checkpoints, used
        return out

    @staticmethod
    def backward(ctx, qbar_out):
        fv, steps, every = ctx.fv, ctx.steps, ctx.every
        qbar = qbar_out.detach().to(torch.float64).contiguous().clone()
        starts = sorted(ctx.checkpoints)
        for k in reversed(range(len(starts))):
            first = starts[k]
            last = starts[k + 1] if k + 1 < len(starts) else steps
            fv.set_state(ctx.checkpoints[first])
            states = []
            for s in range(first, last):
                states.append(fv.get_state(torch.empty_like(qbar)))
                if s + 1 < last:
                    fv.time_step(ctx.courant)
                    fv.step(ctx.dts[s])
            for s in reversed(range(first, last)):
                fv.set_state(states[s - first])
                fv.step_adjoint(ctx.dts[s], qbar)
        return qbar, None, None, None, None, None


def rollout(q0, fv: "hydro.FiniteVolume", steps: int, courant: float = 0.3, every: int = 20, dts=None):
    """Q after ``steps`` steps from ``q0``, differentiable in ``q0``."""
    return Rollout.apply(q0, fv, steps, courant, every, dts)


def last_dts(result) -> list:
    """The dt schedule the forward of ``result`` took."""
    fn = result.grad_fn
    return list(fn.dts) if fn is not None and hasattr(fn, "dts") else []


def shear_layer_torch(centres, volume, coefficients, gamma=5.0 / 3.0):
    """The 2D shear layer (rho 2, vx +0.5 for |y - 1/2| < 1/4; rho 1, vx -0.5 elsewhere; p 2.5; vy = 0.01 sum_k a_k
    sin(2 pi k x)) as extensive Q, differentiable in the coefficients a_k."""
    x, y = centres[:, 0], centres[:, 1]
    inner = (y - 0.5).abs() < 0.25
    rho = torch.where(inner, torch.full_like(x, 2.0), torch.full_like(x, 1.0))
    vx = torch.where(inner, torch.full_like(x, 0.5), torch.full_like(x, -0.5))
    k = torch.arange(1, coefficients.shape[0] + 1, dtype=torch.float64, device=x.device)
    vy = 0.01 * (coefficients[None, :] * torch.sin(2 * torch.pi * k[None, :] * x[:, None])).sum(1)
    p = torch.full_like(x, 2.5)
    E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)
    U = torch.stack([rho, rho * vx, rho * vy, E], 1)
    return U * volume[:, None]


def kinetic_y(q):
    """The objective of the adjoint configuration: int rho vy^2 dA = sum_i Q_my^2 / Q_m."""
    return (q[:, 2] * q[:, 2] / q[:, 0]).sum()
