"""Gradients through implicit time steps: the discrete adjoint on the GPU.

The reference has no differentiation; this module differentiates its
discrete step.  A converged step F = Phi(f) satisfies G(F, f) = 0 (the step
residual with the Hamiltonian recomputed from the moments); the gradient of a
loss with respect to f follows from the one with respect to F by one
transpose solve with the coupled Jacobian (``vv_step_adjoint``).  Long runs
keep a checkpoint every `every` steps and recompute each segment during the
backward sweep, so memory is (N/every + every) fields.

    adj = Adjoint(run)                 # an FP64 Run (its context and options)
    gf  = adj.step(F, f, gF)           # one step
    g0  = trajectory_grad(run, f0, 200, every=20, loss="field_energy")
    fN  = VlasovSteps.apply(f0, run, 200, 20)   # torch.autograd.Function
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib


class Adjoint:
    """Adjoint solves on the context of an FP64 ``Run``."""

    def __init__(self, run, rtol=1e-12, atol=1e-50, max_it=3000, restart=30):
        if run.ctx.precision != "fp64":
            raise ValueError("the adjoint needs an FP64 run")
        self.run = run
        self.ctx = run.ctx
        self.opts = _lib.vv_ksp_opts(rtol=rtol, atol=atol, dtol=1e5, max_it=max_it, restart=restart)
        self.last = None

    def step(self, F, f, gF, h2p=None, h2h=None):
        """Gradient with respect to f^n of a loss with gradient gF with respect
        to f^{n+1} = F, for the converged step f -> F."""
        ctx = self.ctx
        gf = torch.empty_like(gF)
        res = _lib.vv_ksp_result()
        xp = lambda t: None if t is None else ctx.xprof(t)
        ctx.call("vv_step_adjoint", ctx.field(F), ctx.field(f), xp(h2p), xp(h2h), ctx.field(gF), ctx.field(gf),
                 C.byref(self.opts), C.byref(res))
        self.last = {"its": res.its, "reason": res.reason, "rnorm": res.rnorm}
        if res.reason < 0:
            raise RuntimeError("adjoint GMRES did not converge (reason %d, %d its)" % (res.reason, res.its))
        return gf

    def field_energy_grad(self, f):
        """dW/df of the field energy W = 1/2 charge sum (phi_{i+1} - phi_i)^2 / hx."""
        g = torch.empty_like(f)
        self.ctx.call("vv_field_energy_grad", self.ctx.field(f), self.ctx.field(g))
        return g


def _set_state(run, f):
    run.fc.copy_(f)
    run.calculate_moments()


def trajectory(run, f0, nsteps, every):
    """Advance from f0 by nsteps; returns (f_N, checkpoints at steps 0, every, ...)."""
    _set_state(run, f0)
    cps = {}
    for k in range(nsteps):
        if k % every == 0:
            cps[k] = run.fc.clone()
        run.step()
    return run.fc.clone(), cps


def trajectory_backward(run, cps, nsteps, every, gN, adj=None):
    """Pull gN (gradient with respect to f_N) back to f_0 through the steps,
    recomputing each segment from its checkpoint."""
    adj = adj or Adjoint(run)
    g = gN
    stats = {"steps": 0, "adjoint_its": 0}
    for k0 in sorted(cps, reverse=True):
        k1 = min(k0 + every, nsteps)
        _set_state(run, cps[k0])
        seg = [run.fc.clone()]
        for _ in range(k0, k1):
            run.step()
            seg.append(run.fc.clone())
        for j in range(len(seg) - 1, 0, -1):
            g = adj.step(seg[j], seg[j - 1], g)
            stats["steps"] += 1
            stats["adjoint_its"] += adj.last["its"]
    return g, stats


def trajectory_grad(run, f0, nsteps, every=20, loss="field_energy", adj=None):
    """Value and gradient with respect to f0 of a loss of f_N (the field
    energy by default, or a callable f_N -> (value, gradient))."""
    adj = adj or Adjoint(run)
    fN, cps = trajectory(run, f0, nsteps, every)
    if loss == "field_energy":
        value = run.invariants()["field_energy"]
        gN = adj.field_energy_grad(fN)
    else:
        value, gN = loss(fN)
    g0, stats = trajectory_backward(run, cps, nsteps, every, gN, adj)
    return value, g0, stats


class VlasovSteps(torch.autograd.Function):
    """f_N = Phi^N(f_0) with the checkpointed discrete adjoint as backward."""

    @staticmethod
    def forward(ctx, f0, run, nsteps, every=20):
        fN, cps = trajectory(run, f0.detach(), nsteps, every)
        ctx.run, ctx.cps, ctx.nsteps, ctx.every = run, cps, nsteps, every
        return fN

    @staticmethod
    def backward(ctx, gN):
        g0, _ = trajectory_backward(ctx.run, ctx.cps, ctx.nsteps, ctx.every, gN.contiguous())
        return g0, None, None, None


__all__ = ["Adjoint", "trajectory", "trajectory_backward", "trajectory_grad", "VlasovSteps"]
