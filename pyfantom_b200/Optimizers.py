"""Optimality-criteria optimizer (drop-in for pyFANTOM/Optimizers/CUDA/OC.py:6-192 and
Optimizers/_optimizer.py).

``OC.iter()`` computes ``ocP = x sqrt(max(-df/dg, 0))`` and bisects the Lagrange
multiplier with the reference's initial bracket [1e-9, 1e9], midpoint rule and stopping
test ``(l2-l1)/(l2+l1) <= 1e-8``; the bisection runs on the device (``pf_oc_update_f64``,
five bisection levels per sweep over the elements, no host round trip per step).
``converged()`` and ``logs()`` keep the reference keys.
"""
from __future__ import annotations

import ctypes
import time

import torch

from . import _lib
from ._tensor import device

__all__ = ["Optimizer", "OC"]


class Optimizer:
    """Optimizer base (pyFANTOM/Optimizers/_optimizer.py:4-32)."""

    def __init__(self, problem, *args, **kwargs):
        self.problem = problem
        self.desvars = problem.init_desvars()

    def iter(self, *args, **kwargs):
        raise NotImplementedError("iter method must be implemented in subclasses.")

    def converged(self, *args, **kwargs):
        raise NotImplementedError("converged method must be implemented in subclasses.")


class OC(Optimizer):
    def __init__(self, problem, move: float = 0.2, change_tol=1e-4, fun_tol=1e-6, timer=False):
        super().__init__(problem)
        if not problem.is_independent():
            raise ValueError("OC optimizer requires a problem with independent constraints.")
        if problem.m() != 1:
            raise NotImplementedError("OC here supports a single volume constraint")
        self.last_desvars = problem.get_desvars().clone()
        self.last_f = problem.f()
        self.m = problem.m()
        self.lambda_map = problem.constraint_map()
        self.move = move
        self.bounds = problem.bounds()
        self.change = float("inf")
        self.change_f = float("inf")
        self.change_tol = change_tol
        self.fun_tol = fun_tol
        self.timer = timer
        self.iteration = 0
        self._work = None
        self.last_lambda = None
        self.last_steps = None

    def _oc_step(self, x, df, dg, vf):
        n = x.shape[0]
        lib = _lib.load()
        if self._work is None or self._work.numel() < lib.pf_oc_workspace_size(n):
            self._work = torch.empty(int(lib.pf_oc_workspace_size(n)), dtype=torch.float64, device=device())
        x_new = torch.empty_like(x)
        out = (ctypes.c_double * 3)()
        df, dg = df.contiguous(), dg.contiguous()  # keep the operands alive across the call
        _lib.check(lib.pf_oc_update_f64(n, _lib.ptr(x), _lib.ptr(df), _lib.ptr(dg),
                                        float(vf), float(self.move), _lib.ptr(x_new), _lib.ptr(self._work), out,
                                        _lib.stream()))
        return x_new, out[0], out[1], int(out[2])

    def iter(self):
        if self.timer:
            start = time.time()
        p = self.problem
        x = p.get_desvars()
        vf = p.volume_fraction
        x_new, change, lam, steps = self._oc_step(x, p.nabla_f(), p.nabla_g(), vf)
        self.last_lambda, self.last_steps = lam, steps
        self.iteration += 1
        if self.timer:
            end = time.time()
        p.set_desvars(x_new)
        self.change = float(torch.linalg.norm(self.last_desvars - x_new))
        f = p.f()
        self.change_f = float(torch.abs((f - self.last_f) / f))
        self.last_f = f
        self.last_desvars = x_new.clone()
        if self.timer:
            return end - start

    def converged(self, *args, **kwargs):
        if not self.problem.is_terminal():
            return False
        return self.change <= self.change_tol and self.change_f <= self.fun_tol

    def logs(self):
        return {"objective": float(self.last_f), "variable change": float(self.change),
                "function change": float(self.change_f), **self.problem.logs()}
