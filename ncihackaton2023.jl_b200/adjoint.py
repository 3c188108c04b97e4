"""Adjoint form of the variable-coefficient operator -div(kappa grad u).

``kappa_apply(A, x, kappa)`` is y = A(kappa) x as a differentiable torch
function, the counterpart of a ChainRulesCore ``rrule`` for the reference's
``mul!``. Its backward pass gives:
* x_bar = A(kappa) y_bar, because A is symmetric;
* kappa_bar[c, q] = (grad y_bar)^T G (grad x) at each point, from the
  device kernel behind sf_kappa_vjp. That kernel recomputes the gradients at
  the points instead of storing them.

``objective_gradient`` is the adjoint-state gradient of
J(kappa) = 0.5 ||u(kappa) - u_obs||^2 with A(kappa) u = b. It takes one
forward CG solve, one adjoint CG solve (A is self-adjoint) and one VJP:
dJ/dkappa = -kappa_bar(x = u, y_bar = lambda), where A lambda = u - u_obs.
"""
from __future__ import annotations

import torch

from .operator import LazyMatrix, cg, mul


class _KappaApply(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, kappa, A):
        A.set_coefficient(kappa)
        y = torch.empty_like(x)
        mul(y, A, x)
        ctx.save_for_backward(x, kappa)
        ctx.A = A
        return y

    @staticmethod
    def backward(ctx, ybar):
        x, kappa = ctx.saved_tensors
        A = ctx.A
        A.set_coefficient(kappa)
        ybar = ybar.contiguous()
        xbar = kbar = None
        if ctx.needs_input_grad[0]:
            xbar = torch.empty_like(ybar)
            mul(xbar, A, ybar)
        if ctx.needs_input_grad[1]:
            kbar = A.kappa_vjp(x, ybar)
        return xbar, kbar, None


def kappa_apply(A: LazyMatrix, x: torch.Tensor, kappa: torch.Tensor) -> torch.Tensor:
    """y = A(kappa) x with gradients with respect to x and kappa (float64 CUDA tensors;
    kappa has shape (ncells, SQ^3))."""
    return _KappaApply.apply(x, kappa, A)


def objective_gradient(A: LazyMatrix, b: torch.Tensor, u_obs: torch.Tensor, kappa: torch.Tensor,
                       reltol: float = 1e-12, mode: str = "jacobi", maxiter: int = 20000):
    """J(kappa) = 0.5 ||u - u_obs||^2 with A(kappa) u = b, and dJ/dkappa by the adjoint
    method. Returns (J, grad (ncells, SQ^3), u, info)."""
    A.set_coefficient(kappa)
    u, i1 = cg(A, b, reltol=reltol, mode=mode, maxiter=maxiter)
    res = u - u_obs
    J = 0.5 * torch.dot(res, res).item()
    lam, i2 = cg(A, res, reltol=reltol, mode=mode, maxiter=maxiter)
    grad = -A.kappa_vjp(u, lam)
    return J, grad, u, {"forward_iters": i1["iters"], "adjoint_iters": i2["iters"]}


def objective(A: LazyMatrix, b: torch.Tensor, u_obs: torch.Tensor, kappa: torch.Tensor,
              reltol: float = 1e-12, mode: str = "jacobi", maxiter: int = 20000) -> float:
    A.set_coefficient(kappa)
    u, _ = cg(A, b, reltol=reltol, mode=mode, maxiter=maxiter)
    r = u - u_obs
    return 0.5 * torch.dot(r, r).item()
