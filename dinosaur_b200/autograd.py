"""torch.autograd.Function wrappers with hand-written adjoint kernels.

The spherical-harmonic transforms are linear; their VJPs are the transposed
transforms (``dino_sht_inverse_adjoint`` / ``dino_sht_forward_adjoint``):
the adjoint of ``to_nodal`` is an unweighted forward Fourier sum followed by
the forward Legendre contraction, and the adjoint of ``to_modal`` is the
inverse contraction followed by Fourier synthesis scaled by the quadrature
weights.  Spectral operators use their transposed kernels.  These are the
maps JAX derives for the reference's einsums
(dinosaur/spherical_harmonic.py:262-280, :1063-1102).
"""

from __future__ import annotations

import torch


class _SHTInverse(torch.autograd.Function):

  @staticmethod
  def forward(ctx, x, plan):
    ctx.plan = plan
    return plan.inverse(x)

  @staticmethod
  def backward(ctx, g):
    return ctx.plan.inverse_adjoint(g.contiguous()), None


class _SHTForward(torch.autograd.Function):

  @staticmethod
  def forward(ctx, z, plan):
    ctx.plan = plan
    return plan.forward(z)

  @staticmethod
  def backward(ctx, g):
    return ctx.plan.forward_adjoint(g.contiguous()), None


class _ModalOp(torch.autograd.Function):

  @staticmethod
  def forward(ctx, x, plan, op, arg):
    ctx.plan, ctx.op, ctx.arg = plan, op, arg
    return plan.modal_op(op, x, arg)

  @staticmethod
  def backward(ctx, g):
    return ctx.plan.modal_op(ctx.op, g.contiguous(), ctx.arg,
                             transpose=True), None, None, None


def _needs_grad(x):
  return torch.is_grad_enabled() and x.requires_grad


def sht_inverse(plan, x):
  return _SHTInverse.apply(x, plan) if _needs_grad(x) else plan.inverse(x)


def sht_forward(plan, z):
  return _SHTForward.apply(z, plan) if _needs_grad(z) else plan.forward(z)


def modal_op(plan, op, x, arg=0, radius=1.0):
  del radius  # scaling is applied by the caller
  if _needs_grad(x):
    return _ModalOp.apply(x, plan, op, arg)
  return plan.modal_op(op, x, arg)
