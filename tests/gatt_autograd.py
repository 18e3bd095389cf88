"""torch.autograd.Function wrappers of the tangent-linear and adjoint entry points.

TEST HARNESS ONLY: the product path is the C-ABI (``gatt_rhs``, ``gatt_run`` and their
``gatt_rhs_jvp`` / ``gatt_rhs_vjp`` / ``gatt_jvp`` / ``gatt_vjp`` linearisations); these
Functions let torch's own machinery -- ``gradcheck``, forward-mode duals, ``autograd.grad``
-- drive those entry points, so that the hand-written tangent and adjoint kernels are
checked by tools that know nothing about them.

A state is a flat float64 tensor of 5 * npts values: U, V, W, R, E one after the other, each
in Fortran (x fastest) order -- the layout the entry points take.
"""
from __future__ import annotations

import numpy as np
import torch


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64, copy=False)


def _t(a, like):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=torch.float64, device=like.device)


class RHS(torch.autograd.Function):
    """q -> F(q), the Navier-Stokes right-hand side (``gatt_rhs``, nseq.F90:142-323).
    Reverse mode: F'(q)^T a (``gatt_rhs_vjp``); forward mode: F'(q) dq (``gatt_rhs_jvp``)."""

    @staticmethod
    def forward(q, g):
        return _t(g._pack(g.nseq(g._unpack(_np(q)))), q)

    @staticmethod
    def setup_context(ctx, inputs, output):
        q, g = inputs
        ctx.g = g
        ctx.save_for_backward(q)
        ctx.save_for_forward(q)

    @staticmethod
    def backward(ctx, a):
        (q,) = ctx.saved_tensors
        g = ctx.g
        return _t(g._pack(g.rhs_vjp(g._unpack(_np(q)), g._unpack(_np(a)))), a), None

    @staticmethod
    def jvp(ctx, dq, _g):
        (q,) = ctx.saved_tensors
        g = ctx.g
        return _t(g._pack(g.rhs_jvp(g._unpack(_np(q)), g._unpack(_np(dq)))), dq)


class Steps(torch.autograd.Function):
    """q0 -> q(nsteps), the time stepper (``gatt_upload`` + ``gatt_run`` + ``gatt_download``:
    RK4, filter and boundary conditions per step, main.F90:306-410).  Reverse mode: the
    checkpointed adjoint (``gatt_vjp``, a checkpoint every `every` steps); forward mode: the
    tangent-linear run (``gatt_jvp``)."""

    @staticmethod
    def forward(q0, g, nsteps, t0, dt, every):
        g.upload(g._unpack(_np(q0)))
        g.run(nsteps, t0, dt)
        return _t(g._pack(g.download()), q0)

    @staticmethod
    def setup_context(ctx, inputs, output):
        q0, g, nsteps, t0, dt, every = inputs
        ctx.g, ctx.args = g, (nsteps, t0, dt, every)
        ctx.save_for_backward(q0)
        ctx.save_for_forward(q0)

    @staticmethod
    def backward(ctx, lam):
        (q0,) = ctx.saved_tensors
        g = ctx.g
        nsteps, t0, dt, every = ctx.args
        g.upload(g._unpack(_np(q0)))
        lam0 = g.vjp(g._unpack(_np(lam)), nsteps, t0, dt, checkpoint_every=every)
        return _t(g._pack(lam0), lam), None, None, None, None, None

    @staticmethod
    def jvp(ctx, dq0, *_):
        (q0,) = ctx.saved_tensors
        g = ctx.g
        nsteps, t0, dt, _every = ctx.args
        g.upload(g._unpack(_np(q0)))
        return _t(g._pack(g.jvp(g._unpack(_np(dq0)), nsteps, t0, dt)), dq0)
