"""Optimality-criteria optimizer (drop-in for pyFANTOM/Optimizers/CUDA/OC.py:6-192 and
Optimizers/_optimizer.py).

``OC.iter()`` computes ``ocP = x sqrt(max(-df/dg, 0))`` and bisects the Lagrange
multiplier with the reference's initial bracket [1e-9, 1e9], midpoint rule and stopping
test ``(l2-l1)/(l2+l1) <= 1e-8``; the bisection runs on the device (``pf_oc_update_f64``,
five bisection levels per sweep over the elements, no host round trip per step).  With
one volume constraint per material the multipliers are bisected in lockstep as in the
reference (``pf_oc_update_multi_f64``).
``converged()`` and ``logs()`` keep the reference keys.
"""
from __future__ import annotations

import ctypes
import math
import sys
import time

import numpy as np
import torch

from . import _lib
from ._tensor import device

__all__ = ["Optimizer", "OC", "PGD"]


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

    def _oc_step_multi(self, x, df, dg, vf):
        nm = self.m
        ne = x.shape[0] // nm
        lib = _lib.load()
        need = int(lib.pf_oc_multi_workspace_size(ne, nm))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.float64, device=device())
        x_new = torch.empty_like(x)
        out = (ctypes.c_double * 3)()
        dgs = dg.sum(dim=0).contiguous()  # per-variable constraint gradient (OC.py:69-70)
        df = df.contiguous()
        vf_h = (ctypes.c_double * nm)(*[float(v) for v in vf])
        _lib.check(lib.pf_oc_update_multi_f64(ne, nm, _lib.ptr(x), _lib.ptr(df), _lib.ptr(dgs), vf_h,
                                              float(self.move), _lib.ptr(x_new), _lib.ptr(self._work), out,
                                              _lib.stream()))
        return x_new, out[0], out[1], int(out[2])

    def _oc_step(self, x, df, dg, vf):
        if self.m > 1:
            return self._oc_step_multi(x, df, dg, vf)
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
        vf = p.volume_fraction if p.is_single_material else p._vf_h
        x_new, change, lam, steps = self._oc_step(x, p.nabla_f(), p.nabla_g(), vf)
        self.last_lambda, self.last_steps = lam, steps
        self.iteration += 1
        if self.timer:
            end = time.time()
        p.set_desvars(x_new)
        # ||x_new - x|| from the update kernel: x is the design the previous iteration set
        # (the reference takes ||last_desvars - desvars_new||, OC.py:137)
        self.change = change
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


class PGD(Optimizer):
    """Projected gradient descent (drop-in for pyFANTOM/Optimizers/CUDA/PGD.py:6-372).

    Same constructor arguments, ``iter``, ``converged`` and ``logs`` as the reference.  One
    iteration: a Barzilai-Borwein step size from the gradient history with the reference's
    safeguards and fall-backs (PGD.alpha, :107-142), optionally along conjugate directions
    (beta = max(dx_n.(dx_n - dx_n-1) / |dx_n-1|^2, 0) with dx = -df), the step
    x + alpha d, then the projection onto the volume constraints by the reference's
    bisection for the shifts l of clip(x + l dg, 0, 1) (:144-170).  The vector work runs in
    the library (``pf_pgd_stats_f64``: the eight dot products and maxima of the step-size
    rule in one pass; ``pf_pgd_step_f64``; ``pf_pgd_project_f64`` /
    ``pf_pgd_project_multi_f64``: the bisection on the device, five levels per pass); the
    scalar rule is evaluated on the host exactly as written in the reference.

    The projection is the reference's ``is_independent or m == 1`` branch, which every
    MinimumCompliance problem takes (``is_independent()`` is always true there): one
    constraint, or one per material with the m shifts bisected in lockstep.  The m > 1
    case needs constraint rows that are zero off their own block of the design, as
    MinimumCompliance builds them.  The Newton / Wolfe-line-search branch for coupled
    constraints (:172-210) serves problems whose ``is_independent()`` is false; no problem
    of this library is one, and such a problem raises NotImplementedError.
    """

    def __init__(self, problem, change_tol=1e-4, fun_tol=1e-6, maxiter_N=50, tol_B=1e-8, tol_N=1e-6, C=1e12,
                 fall_back_move=0.2, alpha_max=1e2, relaxation=1.0, warmup_iter=50, timer=False,
                 conjugate_directions=True):
        super().__init__(problem)
        self.last_desvars = problem.get_desvars().clone()
        self.last_f = problem.f()
        self.last_nabla_f = problem.nabla_f().clone()
        self.m = problem.m()
        self.is_independent = problem.is_independent()
        if self.m > 1 and not self.is_independent:
            raise NotImplementedError("PGD here projects onto independent constraints (problem.is_independent())")
        if self.m > 8:
            raise NotImplementedError("PGD here projects onto at most 8 volume constraints")
        self._blocks = None  # (dg, rows of dg on their own blocks) for m > 1
        self.lambda_map = problem.constraint_map()
        self.bounds = problem.bounds()
        self.change = float("inf")
        self.change_f = float("inf")
        self.change_tol = change_tol
        self.fun_tol = fun_tol
        self.tol_B = tol_B
        self.tol_N = tol_N
        self.C = C
        self.fall_back_move = fall_back_move
        self.alpha_max = alpha_max
        self.maxiter_N = maxiter_N
        self.timer = timer
        self.relaxation = relaxation
        self.warmup_iter = warmup_iter
        self.conjugate = conjugate_directions
        self.iteration = 0
        self.d_last = None
        self.last_alpha = None
        self.last_projection = None
        self._work = None
        desvars = problem.get_desvars()
        dg = problem.nabla_g()
        problem.set_desvars(self.project_to_feasible(desvars.clone(), desvars, dg))

    def _ws(self, n):
        lib = _lib.load()
        need = int(lib.pf_pgd_workspace_size(n))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.float64, device=device())
        return self._work

    def _stats(self, desvars, df, history):
        n = desvars.shape[0]
        out = (ctypes.c_double * 8)()
        xl = self.last_desvars if history else None
        dfl = self.last_nabla_f if history else None
        _lib.check(_lib.load().pf_pgd_stats_f64(n, _lib.ptr(desvars), _lib.ptr(df), _lib.ptr(xl), _lib.ptr(dfl),
                                                _lib.ptr(self._ws(n)), out, _lib.stream()))
        return list(out)

    @staticmethod
    def _nan_to_num(v):
        if math.isnan(v):
            return 0.0
        if math.isinf(v):
            return sys.float_info.max if v > 0 else -sys.float_info.max
        return v

    def alpha(self, desvars, df):
        """(alpha, beta): the step size and the conjugate-direction weight (None: d = -df)."""
        hist = self.iteration > 0
        dfdf, dfmax, dfdl, dldl, sy, ss, yy, ymax = self._stats(desvars, df, hist)
        beta = None
        if self.conjugate and self.iteration > 0:
            # dx_n = -df, dx_n-1 = -df_last: dx_n.(dx_n - dx_n-1) = df.df - df.df_last
            beta = max((dfdf - dfdl) / dldl, 0.0)
        if self.iteration == 0:
            alpha = self.fall_back_move / dfmax
        elif float(self.problem.g().max()) > self.tol_N and self.iteration > self.warmup_iter:
            alpha = self.fall_back_move / dfmax
        else:
            if sy > 1e-6:
                alpha = ss / sy
                L = self._nan_to_num(math.sqrt(yy) / math.sqrt(ss) if ss > 0 else (math.nan if yy == 0 else math.inf))
                alpha = min(max(alpha, 1e-6), min(2 * self.relaxation / (L + 1e-6), self.alpha_max))
            else:
                if ymax <= 1e-8:  # np.allclose(y, 0): perfect linear behaviour
                    L = math.sqrt(dfdf) * (math.sqrt(ss) / math.sqrt(self.problem.N()))
                    alpha = self.relaxation / (L + 1e-6)
                else:
                    L = self._nan_to_num(math.sqrt(yy) / math.sqrt(ss) if ss > 0 else math.inf)
                    alpha = min(self.relaxation / (L + 1e-6), self.alpha_max)
        return alpha, beta

    def project_to_feasible(self, desvars_new, desvars, dg):
        n = desvars_new.shape[0]
        desvars_new = desvars_new.contiguous()
        x_new = torch.empty_like(desvars_new)
        if self.m > 1:
            return self._project_blocks(desvars_new, dg, x_new)
        out = (ctypes.c_double * 3)()
        dg = dg.contiguous()
        _lib.check(_lib.load().pf_pgd_project_f64(n, _lib.ptr(desvars_new), _lib.ptr(dg),
                                                  float(self.problem.volume_fraction), float(self.bounds[0]),
                                                  float(self.bounds[1]), float(self.tol_B), _lib.ptr(x_new),
                                                  _lib.ptr(self._ws(n)), out, _lib.stream()))
        self.last_projection = {"l": out[0], "steps": int(out[1]), "feasible_at_zero": bool(out[2])}
        return x_new

    def _project_blocks(self, desvars_new, dg, x_new):
        """m volume constraints, row i of dg nonzero only on block i of the design."""
        m = self.m
        n = desvars_new.shape[0]
        ne = n // m
        if dg.dim() != 2 or tuple(dg.shape) != (m, n) or ne * m != n:
            raise ValueError(f"nabla_g of shape {tuple(dg.shape)} for {m} constraints on {n} variables")
        if self._blocks is None or self._blocks[0] is not dg:
            rows = torch.stack([dg[i, i * ne:(i + 1) * ne] for i in range(m)]).contiguous()
            if int(torch.count_nonzero(dg)) != int(torch.count_nonzero(rows)):
                raise NotImplementedError("PGD here projects onto constraints with block-diagonal rows "
                                          "(one volume constraint per material)")
            self._blocks = (dg, rows)
        rows = self._blocks[1]
        vf = getattr(self.problem, "_vf_h", None)
        if vf is None:
            vf = self.problem.volume_fraction
            vf = vf.cpu() if torch.is_tensor(vf) else vf
        vf = np.broadcast_to(np.asarray(vf, dtype=np.float64), (m,)).copy()
        lib = _lib.load()
        need = int(lib.pf_pgd_multi_workspace_size(ne, m))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.float64, device=device())
        out = (ctypes.c_double * (2 + m))()
        _lib.check(lib.pf_pgd_project_multi_f64(ne, m, _lib.ptr(desvars_new), _lib.ptr(rows),
                                                vf.ctypes.data_as(ctypes.c_void_p), float(self.bounds[0]),
                                                float(self.bounds[1]), float(self.tol_B), _lib.ptr(x_new),
                                                _lib.ptr(self._work), out, _lib.stream()))
        self.last_projection = {"l": list(out[2:2 + m]), "steps": int(out[0]), "feasible_at_zero": bool(out[1])}
        return x_new

    def iter(self):
        if self.timer:
            start = time.time()
        p = self.problem
        desvars = p.get_desvars()
        dg = p.nabla_g()
        df = p.nabla_f().clone()
        f = p.f()
        alpha, beta = self.alpha(desvars, df)
        n = desvars.shape[0]
        d = torch.empty_like(desvars)
        x_step = torch.empty_like(desvars)
        d_last = self.d_last if beta is not None else None
        _lib.check(_lib.load().pf_pgd_step_f64(n, _lib.ptr(desvars), _lib.ptr(df), _lib.ptr(d_last),
                                               float(beta if beta is not None else 0.0), float(alpha), _lib.ptr(d),
                                               _lib.ptr(x_step), _lib.stream()))
        self.last_alpha = alpha
        self.last_nabla_f = df
        self.d_last = d
        self.last_desvars = desvars.clone()
        self.last_f = f
        self.iteration += 1
        desvars_new = self.project_to_feasible(x_step, desvars, dg)
        if self.timer:
            end = time.time()
        p.set_desvars(desvars_new)
        self.change = float(torch.linalg.norm(self.last_desvars - desvars_new))
        fn = p.f()
        self.change_f = float(abs((fn - self.last_f) / fn))
        if self.timer:
            return end - start

    def converged(self, *args, **kwargs):
        if not self.problem.is_terminal():
            return False
        return self.change <= self.change_tol and self.change_f <= self.fun_tol

    def logs(self):
        return {"objective": float(self.last_f), "variable change": float(self.change),
                "function change": float(self.change_f), **self.problem.logs()}
