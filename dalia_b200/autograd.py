"""``torch.autograd`` interface of the INLA objective.

The reference differentiates its objective f(theta) = -log pi(theta | y)
(up to a constant) by central finite differences: 2 dim(theta) + 1 further
evaluations of f, each with its own factorisations
(``DALIA._objective_function``, ``src/dalia/core/dalia.py:513-601``; the
loop over the stencil is ``:548-581``).  Here f is a differentiable torch
function instead:

* ``forward`` assembles Q_conditional(theta) and Q_prior(theta) on the
  device, factorises both (batched over all points), computes the log-
  determinants and the latent mean, and returns f -- everything the
  reference's f evaluation does;
* ``backward`` runs the selected inversions of both matrices and the
  contraction kernels: tr(Q^{-1} dQ/dtheta) from block inner products of the
  selected inverse with the Kronecker factors of dQ/dtheta (recomputed from
  the O(nt) scalar coefficients, never stored), the quadratic and likelihood
  terms from the forward's latent mean, and for a Poisson likelihood the
  implicit term through the mode; it returns grad_out * grad f.

``theta`` of shape (d,) gives a scalar f; shape (K, d) evaluates K points in
one batch (all 2K factorisations and selected inversions share their
launches) and gives f of shape (K,).  The forward's device state lives in the
model; a second forward before the first one's backward overwrites it, and
that backward then recomputes its forward first.
"""

from __future__ import annotations

import numpy as np
import torch
from torch.autograd.function import once_differentiable


class NegLogPosterior(torch.autograd.Function):
    """f(theta) with the adjoint gradient as its backward (see the module
    docstring).  Use through ``objective``."""

    @staticmethod
    def forward(ctx, theta, model, precision):
        th = theta.detach().to("cpu", torch.float64).numpy()
        if th.ndim not in (1, 2) or th.shape[-1] != len(model.theta_keys):
            raise ValueError(f"theta must have shape (d,) or (K, d) with d = {len(model.theta_keys)}")
        tok = model.adjoint_forward(list(th.reshape(-1, th.shape[-1])), precision, check=True)
        ctx.model, ctx.tok, ctx.shape = model, tok, tuple(theta.shape)
        f = model.f_device(tok).to(device=theta.device, dtype=theta.dtype)
        return f if th.ndim == 2 else f[0]

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_out):
        _, grads = ctx.model.adjoint_backward(ctx.tok)
        G = torch.as_tensor(np.stack(grads), dtype=grad_out.dtype, device=grad_out.device)
        if len(ctx.shape) == 1:
            return grad_out * G[0], None, None
        return grad_out[:, None] * G, None, None


def objective(model, theta, precision=None):
    """f(theta) = -log pi(theta | y) + const of a ``SpatioTemporalModel`` or
    ``CoregionalModel`` as a differentiable tensor (the reference's
    objective, ``dalia.py:603-745``).  ``precision`` selects the arithmetic
    of the selected inversions behind the gradient ("fp64", "i8slice",
    "tf32x3"; default: the model's), with the model's per-point accuracy
    check and FP64 fallback."""
    return NegLogPosterior.apply(theta, model, precision)
