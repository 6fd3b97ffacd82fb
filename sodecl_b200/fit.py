"""Model fitting: loss and gradients of trajectories w.r.t. parameters and y0.

    sim = Integrator(system_path("oculomotor"), "rk4", dt=1e-5, tspan=0.05, ksteps=100,
                     neq=6, npar=6, orbits=n)
    adj = Adjoint(sim)
    loss = trajectory_mse(params, y0, t0, targets, adj)   # torch tensors on the GPU
    loss.sum().backward()                                  # params.grad, y0.grad

Per orbit i, loss_i = sum_{r,e} (y_{r,e,i} - target_{r,e,i})^2 / (records * neq)
over the records the integrator's configuration produces.  The gradient is the
discrete adjoint of the Euler/RK4 steps, and of the implicit Euler/midpoint
steps through their transposed Newton systems (sodecl_cuda_adjoint), computed on the
GPU by one kernel; `finite_difference_gradient` is the central-difference
baseline on the same GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


def _torch():
    import torch

    return torch


class Adjoint:
    def __init__(self, integrator, ckpt_every=0, tape_entries=256, use_tape=False):
        """use_tape: differentiate sode_system on the reverse-mode tape even if
        the system file provides calc_jacobian and calc_jacobian_params."""
        self.sim = integrator
        self.ckpt_every = int(ckpt_every)
        self.tape_entries = int(tape_entries)
        self.use_tape = bool(use_tape)

    def __call__(self, t0, y0, params, targets, with_gradient=True):
        """(loss[n], grad_params[n,npar] or None, grad_y0[n,neq] or None, flags[n])
        for device tensors t0[n], y0[n,neq], params[n,npar], targets[records,neq,n]."""
        torch = _torch()
        n = t0.numel()
        dev = t0.device
        f64 = torch.float64
        t0, y0, params, targets = (x.detach().to(f64).contiguous() for x in (t0, y0, params, targets))
        if targets.shape != (self.sim.num_records, self.sim.neq, n):
            raise ValueError("targets must be (records, neq, orbits) = %s" % ((self.sim.num_records, self.sim.neq, n),))
        loss = torch.empty(n, dtype=f64, device=dev)
        gp = torch.empty((n, self.sim.cfg.num_params), dtype=f64, device=dev) if with_gradient else None
        gy = torch.empty((n, self.sim.neq), dtype=f64, device=dev) if with_gradient else None
        flags = torch.zeros(n, dtype=torch.int32, device=dev)
        io = N.AdjointIO()
        io.t0, io.y0, io.params, io.targets = t0.data_ptr(), y0.data_ptr(), params.data_ptr(), targets.data_ptr()
        io.loss = loss.data_ptr()
        io.grad_params = gp.data_ptr() if gp is not None else None
        io.grad_y0 = gy.data_ptr() if gy is not None else None
        io.flags = flags.data_ptr()
        io.n = n
        io.ckpt_every = self.ckpt_every
        io.tape_entries = self.tape_entries
        io.use_tape = 1 if self.use_tape else 0
        stream = torch.cuda.current_stream(dev).cuda_stream
        N.check(N.lib.sodecl_cuda_adjoint(self.sim.ctx, C.byref(io), stream), self.sim.ctx)
        return loss, gp, gy, flags


def _function():
    torch = _torch()

    class TrajectoryMSE(torch.autograd.Function):
        """loss[n] = per-orbit MSE of the trajectory from (params, y0) against targets."""

        @staticmethod
        def forward(ctx, params, y0, t0, targets, adjoint):
            loss, gp, gy, flags = adjoint(t0, y0, params, targets, with_gradient=True)
            if int((flags != 0).sum()):
                raise RuntimeError("adjoint tape overflow: raise Adjoint(tape_entries=...)")
            ctx.save_for_backward(gp, gy)
            return loss

        @staticmethod
        def backward(ctx, grad_loss):
            gp, gy = ctx.saved_tensors
            g = grad_loss.to(gp.dtype)[:, None]
            return g * gp, g * gy, None, None, None

    return TrajectoryMSE


_FN = None


def trajectory_mse(params, y0, t0, targets, adjoint):
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(params, y0, t0, targets, adjoint)


def finite_difference_gradient(t0, y0, params, targets, adjoint_wide, rel_step=1e-6):
    """Central differences of the per-orbit loss w.r.t. every parameter and
    initial value, all 2 x (npar + neq) perturbed copies of every orbit in one
    launch of the loss kernel.  The step of each entry is rel_step x its
    magnitude (rel_step itself for entries that are exactly zero): an absolute
    floor would be far too coarse for small parameters such as the
    oculomotor model's 0.0045 time constant, whose loss curves as 1/p.
    `adjoint_wide` must wrap an integrator sized for n * 2 * (npar + neq)
    orbits.  Returns (grad_params, grad_y0)."""
    torch = _torch()
    n, npar = params.shape
    neq = y0.shape[1]
    k = npar + neq
    theta = torch.cat([params, y0], dim=1)                              # [n, k]
    mag = theta.abs()
    h = rel_step * torch.where(mag > 0, mag, torch.ones_like(mag))       # [n, k]
    eye = torch.eye(k, dtype=theta.dtype, device=theta.device)
    sign = torch.tensor([1.0, -1.0], dtype=theta.dtype, device=theta.device)
    # pert[s, d, i] = theta[i] + sign[s] * h[i, d] * e_d, copies ordered [sign][direction][orbit]
    pert = theta[None, None] + sign[:, None, None, None] * eye[None, :, None, :] * h.T[None, :, :, None]
    pert = pert.reshape(2 * k * n, k)
    rep = lambda x: x.repeat(2 * k, *([1] * (x.dim() - 1)))  # noqa: E731
    tgt = targets.repeat(1, 1, 2 * k)
    loss, _, _, _ = adjoint_wide(rep(t0), pert[:, npar:].contiguous(), pert[:, :npar].contiguous(), tgt,
                                 with_gradient=False)
    loss = loss.reshape(2, k, n)
    # divide by the perturbation the rounded copies actually carry
    up, down = theta.T + h.T, theta.T - h.T                             # [k, n]
    g = (loss[0] - loss[1]) / (up - down)                               # [k, n]
    return g[:npar].T.contiguous(), g[npar:].T.contiguous()
