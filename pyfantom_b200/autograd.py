"""Compliance and volume of a SIMP problem as differentiable torch functions.

``compliance(x, problem)`` returns c(x) = f . U(x) with K(E(H x)) U = f, where H is the
density filter and E the SIMP law of ``problem`` (a ``MinimumCompliance``).  Its backward
is the adjoint of the compliance, which is self-adjoint (the adjoint state is -U):

    dc/dx = H^T [ dE/drho (H x) * (-u_e^T K0 u_e) ]

evaluated by one fused library kernel (``pf_adjoint_f64``: element energy, SIMP derivative
and the product) followed by the filter transpose (``pf_filter_adj_f64``).  This is the
gradient the reference forms in MinimumCompliance._compute
(pyFANTOM/Problem/CUDA/MinimumCompliance.py:413-445) from process_grad, penalize_grad and
filter._rmatvec.

``volume(x, problem)`` returns the volume fraction nabla_g . x (pyFANTOM/Problem/CUDA/
MinimumCompliance.py:522-525 without the target) with gradient nabla_g.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._tensor import as_cuda

__all__ = ["compliance", "volume", "Compliance", "Volume"]


class Compliance(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, problem):
        if not problem.is_single_material:
            raise NotImplementedError("the differentiable compliance covers single-material problems")
        x = as_cuda(x.detach(), torch.float64)
        rho = problem.filter.dot(x)
        E = problem.penalize(rho)
        U, _ = problem.FE.solve(E)
        U = U.clone()  # the solver keeps its warm start in place
        c = torch.dot(problem.FE.rhs, U)
        ctx.problem = problem
        ctx.save_for_backward(U, rho)
        return c

    @staticmethod
    def backward(ctx, grad_c):
        U, rho = ctx.saved_tensors
        p = ctx.problem
        out = torch.empty_like(rho)
        params = p._params()
        _lib.check(_lib.load().pf_adjoint_f64(p.FE.kernel._op, _lib.ptr(U), _lib.ptr(rho), ctypes.byref(params), 1.0,
                                              _lib.ptr(out), _lib.stream()))
        return grad_c * p.filter._rmatvec(out), None


class Volume(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, problem):
        ctx.problem = problem
        return torch.dot(problem.nabla_g(), as_cuda(x.detach(), torch.float64))

    @staticmethod
    def backward(ctx, grad_v):
        return grad_v * ctx.problem.nabla_g(), None


def compliance(x: torch.Tensor, problem) -> torch.Tensor:
    """Differentiable compliance f . U(x) of ``problem`` at design variables ``x``."""
    return Compliance.apply(x, problem)


def volume(x: torch.Tensor, problem) -> torch.Tensor:
    """Differentiable volume fraction of ``problem`` at design variables ``x``."""
    return Volume.apply(x, problem)
