"""A thin torch.autograd.Function over the library's adjoint (the gradient
harness): the loss is the last step's field energy of an nsteps run, as a
differentiable function of the initial velocities and, for a Darwin run with
the whistler pump, of the pump amplitude a (the pump field is a times the
context's pump).

The forward calls aw_grad_es / aw_grad_darwin, which return the loss and its
gradients together (a forward run with checkpoints and the backward sweep, on
the GPU); backward() only scales the stored gradients by the incoming one. No
autograd graph of the simulation is built: torch is the plumbing here.
"""
from __future__ import annotations

import torch

from . import AW_MODEL_DARWIN, AW_MODEL_ES


class FieldEnergyRun:
    """A context with bound particle tensors x, y, ux, uy, uz, w (cell units) whose
    x, y, w hold the initial state; u0 is supplied per call."""

    def __init__(self, ctx, parts: dict, nsteps: int, checkpoint_every: int, pump: dict | None = None):
        self.ctx, self.parts, self.nsteps, self.every = ctx, parts, int(nsteps), int(checkpoint_every)
        self.pump = dict(pump) if pump else None
        if ctx.model not in (AW_MODEL_ES, AW_MODEL_DARWIN):
            raise ValueError("field-energy gradients need an electrostatic or Darwin context")


class _FieldEnergy(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u0, amplitude, run):
        ctx, P = run.ctx, run.parts
        with torch.no_grad():
            P["ux"].copy_(u0[:, 0])
            P["uy"].copy_(u0[:, 1])
            P["uz"].copy_(u0[:, 2])
        du = [torch.zeros_like(P["ux"]) for _ in range(3)]
        torch.cuda.current_stream(P["ux"].device).synchronize()
        if ctx.model == AW_MODEL_DARWIN:
            a = float(amplitude)
            prm = ctx.params
            if run.pump:
                if a == 0.0:
                    raise ValueError("pump amplitude 0: the gradient is taken relative to the pump's own scale")
                pump = {k: run.pump[k] * (a if k in ("ex", "ey", "ez") else 1.0) for k in run.pump}
                ctx.set_params(dt=prm.dt, qm=prm.qm, eps0=prm.eps0, n0=prm.n0, c=prm.c, B0=tuple(prm.B0),
                               has_b0=bool(prm.has_b0), pump=pump)
            loss, dp = ctx.grad_darwin(run.nsteps, run.every, *du)
            da = dp / a if run.pump else 0.0       # dL/d(a') at a' = 1 of the scaled pump, per unit of a
        else:
            loss = ctx.grad_es(run.nsteps, run.every, *du)
            da = 0.0
        g = torch.stack(du, dim=1)
        fctx.save_for_backward(g)
        fctx.da = da
        return torch.tensor(loss, dtype=torch.float64, device=u0.device)

    @staticmethod
    def backward(fctx, gout):
        (g,) = fctx.saved_tensors
        ga = gout * fctx.da
        return (gout.to(g.dtype) * g, ga.to(torch.float64).reshape(()), None)


def field_energy(run: FieldEnergyRun, u0: torch.Tensor, amplitude: torch.Tensor | None = None) -> torch.Tensor:
    """loss(u0 [n, 3] float32 on the run's device, amplitude a: 0-dim float64
    tensor, 1 = the context's pump) -> 0-dim float64 tensor; differentiable in
    u0 and amplitude."""
    if amplitude is None:
        amplitude = torch.tensor(1.0, dtype=torch.float64, device=u0.device)
    return _FieldEnergy.apply(u0, amplitude, run)
