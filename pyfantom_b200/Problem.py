"""SIMP minimum-compliance problem (drop-in for
pyFANTOM/Problem/CUDA/MinimumCompliance.py:10-635 and Problem/_problem.py).

SIMP with the reference's law: densities are filtered, optionally Heaviside-projected,
penalised as ``E = clip(clip(H(rho)^p, void, 1) * E_mul, void, inf)`` and solved; the
objective is the compliance ``rhs . U`` and its gradient is
``H_filter^T (p H^{p-1} H' E_mul * (-u_e^T K0 u_e))``.  With several materials
(``len(E_mul) > 1``, MinimumCompliance.py:326-349, 369-411) the design variables are
material-major, each material's densities are filtered separately and mixed as
``E = max(sum_i E_mul_i a_i prod_{j != i} (1 - a_j), void)`` with ``a_i = H(rho_i)^p``; there is
one volume constraint per material.  Filtering, penalisation, the element sensitivity and
the adjoint filter run in the library kernels.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Union

import numpy as np
import torch

from . import _lib
from ._tensor import as_cuda, device

__all__ = ["Problem", "MinimumCompliance"]


class Problem:
    """Problem base (pyFANTOM/Problem/_problem.py:1-74)."""

    def ill_conditioned(self, *args, **kwargs):
        return False


def simp_params(penalty, void, E_mul, beta, eta, heavyside) -> _lib.pf_simp_params:
    p = _lib.pf_simp_params()
    p.penalty = float(penalty)
    p.void_value = float(void)
    p.E_mul = float(E_mul)
    p.beta = float(beta)
    p.eta = float(eta)
    p.heavyside = int(bool(heavyside))
    return p


def penalize_device(rho: torch.Tensor, params: _lib.pf_simp_params, want_E=True, want_dE=False):
    rho = as_cuda(rho, torch.float64)
    E = torch.empty_like(rho) if want_E else None
    dE = torch.empty_like(rho) if want_dE else None
    _lib.check(_lib.load().pf_penalize_f64(rho.numel(), _lib.ptr(rho), ctypes.byref(params), _lib.ptr(E),
                                           _lib.ptr(dE), _lib.stream()))
    return E, dE


class MinimumCompliance(Problem):
    def __init__(self, FE, filter, E_mul: list = [1.0], void: float = 1e-6, penalty: float = 3.0,
                 volume_fraction: list = [0.25], penalty_schedule: Callable[[float, int], float] = None,
                 heavyside: bool = True, beta: Union[float, Callable[[int], float]] = 2, eta: float = 0.5):
        if len(E_mul) != len(volume_fraction):
            raise ValueError("E and volume_fraction must have the same length.")
        if len(E_mul) == 1:
            self.is_single_material = True
            self.E_mul = float(E_mul[0])
            self.volume_fraction = float(volume_fraction[0])
            self.n_material = 1
        else:
            if len(E_mul) > 8:
                raise ValueError("at most 8 materials")
            self.is_single_material = False
            self._E_mul_h = np.asarray(E_mul, dtype=np.float64)
            self._vf_h = np.asarray(volume_fraction, dtype=np.float64)
            self.E_mul = torch.as_tensor(self._E_mul_h, device=device())
            self.volume_fraction = torch.as_tensor(self._vf_h, device=device())
            self.n_material = len(E_mul)
        self.void = void
        self.penalty = penalty
        self.penalty_schedule = penalty_schedule
        self.heavyside = heavyside
        self.beta = beta
        self.eta = eta
        self.filter = filter
        self.FE = FE
        self.dtype = FE.dtype
        self.iteration = 0
        self.desvars = None
        self._f = None
        self._g = None
        self._nabla_f = None
        self.nel = int(np.prod(FE.mesh.nel))
        self.num_vars = self.nel * self.n_material
        per_el = (FE.mesh.As / FE.mesh.volume).to(torch.float64)
        if per_el.numel() == 1:
            per_el = per_el.repeat(self.nel)
        if self.is_single_material:
            self._nabla_g = per_el.clone()
        else:
            self._nabla_g = torch.zeros((self.n_material, self.num_vars), dtype=torch.float64, device=device())
            for i in range(self.n_material):
                self._nabla_g[i, i * self.nel:(i + 1) * self.nel] = per_el
        self._residual = None
        self.is_3D = len(FE.mesh.nel) == 3

    def N(self):
        return self.num_vars

    def m(self):
        return self.n_material

    def is_independent(self):
        return True

    def constraint_map(self):
        if self.is_single_material:
            return 1
        mapping = torch.zeros((self.n_material, self.num_vars), dtype=torch.float64, device=device())
        for i in range(self.n_material):
            mapping[i, i * self.nel:(i + 1) * self.nel] = 1
        return mapping

    def bounds(self):
        return (0, 1.0)

    def init_desvars(self):
        v = self.volume_fraction if self.is_single_material else float(self._vf_h.min())
        self.desvars = torch.full((self.num_vars,), v, dtype=torch.float64, device=device())
        self.iteration = 0
        self._compute()

    def set_desvars(self, desvars):
        if desvars.shape[0] != self.num_vars:
            raise ValueError(f"Expected {self.num_vars} design variables, got {desvars.shape[0]}.")
        self.desvars = as_cuda(desvars, torch.float64)
        self._compute()
        self.iteration += 1

    def get_desvars(self):
        return self.desvars

    def _params(self):
        pen = self.penalty
        if self.penalty_schedule is not None:
            pen = self.penalty_schedule(self.penalty, self.iteration)
        beta_val = self.beta(self.iteration) if callable(self.beta) else self.beta
        # the multi-material kernel takes E_mul per material separately
        emul = self.E_mul if self.is_single_material else 1.0
        return simp_params(pen, self.void, emul, beta_val, self.eta, self.heavyside)

    def _penalize_multi(self, rho_mm, want_E=True, want_dE=True):
        """Material-major densities [n_material * nel] -> (E [nel], dE [n_material * nel])."""
        rho_mm = as_cuda(rho_mm, torch.float64)
        E = torch.empty(self.nel, dtype=torch.float64, device=device()) if want_E else None
        dE = torch.empty_like(rho_mm) if want_dE else None
        params = self._params()
        _lib.check(_lib.load().pf_penalize_multi_f64(self.nel, self.n_material, _lib.ptr(rho_mm), ctypes.byref(params),
                                                     self._E_mul_h.ctypes.data, _lib.ptr(E), _lib.ptr(dE),
                                                     _lib.stream()))
        return E, dE

    def penalize(self, rho):
        if self.is_single_material:
            return penalize_device(rho, self._params(), True, False)[0]
        # reference layout [nel, n_material]
        return self._penalize_multi(as_cuda(rho, torch.float64).T.contiguous().reshape(-1), True, False)[0]

    def penalize_grad(self, rho):
        if self.is_single_material:
            return penalize_device(rho, self._params(), False, True)[1]
        dE = self._penalize_multi(as_cuda(rho, torch.float64).T.contiguous().reshape(-1), False, True)[1]
        return dE.reshape(self.n_material, self.nel).T

    def _filtered(self):
        if self.is_single_material:
            return self.filter.dot(self.desvars)
        rho = torch.empty_like(self.desvars)
        for i in range(self.n_material):
            sl = slice(i * self.nel, (i + 1) * self.nel)
            rho[sl] = self.filter.dot(self.desvars[sl].contiguous())
        return rho

    def _compute(self):
        rho = self._filtered()
        if self.is_single_material:
            E, dE = penalize_device(rho, self._params(), True, True)
        else:
            E, dE = self._penalize_multi(rho, True, True)
        U, residual = self.FE.solve(E)
        self._f = torch.dot(self.FE.rhs, U)
        df = self.FE.kernel.process_grad(U)
        if self.is_single_material:
            self._nabla_f = self.filter._rmatvec(dE * df)
        else:
            nf = torch.empty_like(dE)
            for i in range(self.n_material):
                sl = slice(i * self.nel, (i + 1) * self.nel)
                nf[sl] = self.filter._rmatvec((dE[sl] * df).contiguous())
            self._nabla_f = nf
        self._residual = residual
        self._U = U

    def f(self, rho=None):
        if rho is None:
            return self._f
        return self._f + torch.dot(as_cuda(rho, torch.float64), self._nabla_f)

    def nabla_f(self, rho=None):
        return self._nabla_f

    def g(self, rho=None):
        r = self.desvars if rho is None else as_cuda(rho, torch.float64)
        if self.is_single_material:
            return (torch.dot(self._nabla_g, r) - self.volume_fraction).reshape(1)
        return self._nabla_g @ r - self.volume_fraction

    def nabla_g(self):
        return self._nabla_g

    def ill_conditioned(self):
        return self._residual >= 1e-2

    def is_terminal(self):
        if self.penalty_schedule is not None:
            return self.penalty_schedule(self.penalty, self.iteration) == self.penalty
        return True

    def logs(self):
        return {"iteration": int(self.iteration), "residual": float(self._residual)}

    def FEA(self, thresshold: bool = True):
        if self.desvars is None:
            raise ValueError("Design variables are not initialized. Call init_desvars() or set_desvars() first.")
        if thresshold:
            rho = (self.get_desvars() > 0.5).to(torch.float64) + self.void
        else:
            rho = self.get_desvars().clone()
        if self.is_single_material:
            rho = rho * self.E_mul
        else:
            rho = (rho.reshape(self.n_material, -1).T * self.E_mul[None, :]).sum(dim=1)
        solver = self.FE.solver
        if hasattr(solver, "maxiter"):
            solver.maxiter = solver.maxiter * 4
        U, residual = self.FE.solve(rho)
        return {"compliance": torch.dot(self.FE.rhs, U), "Displacements": U}
