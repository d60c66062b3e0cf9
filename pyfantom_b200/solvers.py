"""Linear solvers (drop-in for pyFANTOM/solvers/CUDA/_solvers.py and solvers/commons).

* ``CG``        - matrix-free unpreconditioned CG (reference :22-132), ``pf_cg_solve``.
* ``SPSOLVE``   - direct solve for small problems (reference :245-328): the free-DOF block
  of K assembled dense on the device and factored by the library's tiled Cholesky
  (``pf_direct_solve_f64``, up to 20,480 free DOFs).
* ``MultiGrid`` - geometric-multigrid-preconditioned CG (reference :330-660) with the
  reference's V-cycle (and its lower-case ``cycle='w'`` W-cycle, which repeats the coarse
  correction at the levels in ``w_level``; the default ``'W'`` runs V-cycles there too),
  damped-Jacobi smoother, adaptive omega schedule, Galerkin
  hierarchy and normalised transfers; the coarse solve is a dense Cholesky on the
  device instead of host CHOLMOD (every reference ``coarse_solver`` name maps to it,
  with the same ``beta = 1e-6`` shift).  Keyword-only extras: ``precision`` ('fp64',
  'mixed': FP32 V-cycle inside the FP64 CG, or 'mixed_bf16': the same with the V-cycle's
  fine-level element scales stored as BF16), ``check_every`` (host poll interval) and
  ``warm_start`` (an object with ``guess(kernel, rhs)``, e.g. learned.LearnedWarmStart,
  that supplies the initial guess of a solve that does not reuse ``last_x0``) and
  ``coarse_op`` ('element': level 1 applied element by element from the fine densities
  when the element allows it; 'stencil': assembled stencils on every level; 'auto', the
  default: element by element in the FP32 V-cycle of the mixed forms, where it is faster
  than the FP32 stencil, and the stencil in the FP64 form, where the stencil is faster)
  and ``coarse_correction`` (an object with ``field(kernel, rhs)``, e.g.
  learned.LearnedCoarseSpace, whose nodal field spans a deflation space of the PCG,
  ``pf_mg_set_deflation``) and ``fixed_omega`` (None: the reference's residual-driven
  Jacobi weight, which changes the preconditioner from one iteration to the next; a
  number: that weight in every V-cycle, a fixed preconditioner as PCG assumes).

``solve(rhs, rho=None, use_last=True)`` returns ``(U, residual)`` like the reference;
``last_x0`` holds the warm start.  Solver statistics of the last call are in
``last_info`` (iterations, status, setup/solve milliseconds).
"""
from __future__ import annotations

import ctypes
import logging

import numpy as np
import torch

from . import _lib
from ._tensor import as_cuda, device

__all__ = ["Solver", "CG", "SPSOLVE", "MultiGrid", "SolveInfo"]

logger = logging.getLogger(__name__)


class Solver:
    """Solver base (pyFANTOM/solvers/commons/__init__.py:1-68)."""

    def __call__(self, *args, **kwargs):
        return self.solve(*args, **kwargs)

    def solve(self, *args, **kwargs):
        raise NotImplementedError("solve method must be implemented in subclasses.")

    def reset(self):
        pass


class SolveInfo(dict):
    """iterations, status (name), residual, setup_ms, solve_ms of the last solve."""


def _info(ci: _lib.pf_solve_info) -> SolveInfo:
    return SolveInfo(iterations=ci.iterations, status=_lib.STATUS_NAMES.get(ci.status, str(ci.status)),
                     status_code=ci.status, residual=ci.residual, setup_ms=ci.setup_ms, solve_ms=ci.solve_ms)


class CG(Solver):
    """Matrix-free CG on a StructuredStiffnessKernel (reference _solvers.py:22-132)."""

    def __init__(self, kernel, maxiter=1000, tol=1e-5, matrix_free=None):
        self.kernel = kernel
        self.last_x0 = None
        self.tol = tol
        self.maxiter = maxiter
        self.matrix_free = True if matrix_free is None else matrix_free
        if not self.matrix_free:
            raise NotImplementedError("assembled (matrix_free=False) CG needs CSR assembly, which this library omits")
        self._work = None
        self.last_info = None

    def solve(self, rhs, rho=None, use_last=True):
        k = self.kernel
        if not (k.has_rho or rho is not None):
            raise ValueError("Solver requires a density vector to be passed or set on the kernel.")
        if rho is not None:
            k.set_rho(rho)
        lib = _lib.load()
        rhs = as_cuda(rhs, torch.float64)
        n = rhs.shape[0]
        if self._work is None:
            self._work = torch.empty(int(lib.pf_cg_workspace_size(k._op)), dtype=torch.float64, device=device())
        warm = use_last and self.last_x0 is not None
        x = self.last_x0.clone() if warm else torch.empty(n, dtype=torch.float64, device=device())
        info = _lib.pf_solve_info()
        _lib.check(lib.pf_cg_solve(k._op, _lib.ptr(k.rho), k._mask_ptr(), _lib.ptr(rhs), _lib.ptr(x), int(warm),
                                   float(self.tol), int(self.maxiter), _lib.ptr(self._work), ctypes.byref(info),
                                   _lib.stream()))
        self.last_info = _info(info)
        if use_last:
            self.last_x0 = x
        r = rhs - k.dot(x)
        residual = float(torch.linalg.norm(r) / torch.linalg.norm(rhs))
        return x, residual


class SPSOLVE(Solver):
    """Direct solver (reference _solvers.py:245-328): solves the free DOFs of K(rho) exactly
    (dense Cholesky on the device) and keeps the right-hand side on constrained DOFs."""

    def __init__(self, kernel):
        super().__init__()
        if kernel.shape[0] > 3e6:
            raise ValueError("Currently we do not allow spsolve for problem size bigger than 3M degrees of freedom.")
        self.kernel = kernel
        self.last_x0 = None
        self._h = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.pf_direct_destroy(h)
            self._h = None

    def solve(self, rhs, rho=None, **kwargs):
        k = self.kernel
        if rho is not None:
            k.set_rho(rho)
        elif not k.has_rho:
            raise ValueError("Solver requires a density vector to be passed or set on the kernel.")
        lib = _lib.load()
        if self._h is None:
            h = ctypes.c_void_p()
            _lib.check(lib.pf_direct_create(k._op, ctypes.byref(h)))
            self._h = h
        rhs = as_cuda(rhs, torch.float64)
        free = torch.nonzero(~k.constraints).reshape(-1).to(torch.int32) if k.has_con else \
            torch.arange(rhs.shape[0], dtype=torch.int32, device=device())
        d2f = torch.full((rhs.shape[0],), -1, dtype=torch.int32, device=device())
        d2f[free.long()] = torch.arange(free.numel(), dtype=torch.int32, device=device())
        out = torch.empty_like(rhs)
        _lib.check(lib.pf_direct_solve_f64(self._h, _lib.ptr(k.rho), _lib.ptr(free), _lib.ptr(d2f), int(free.numel()),
                                           _lib.ptr(rhs), _lib.ptr(out), _lib.stream()))
        residual = float(torch.linalg.norm(rhs - k.dot(out)) / torch.linalg.norm(rhs))
        return out, residual


class MultiGrid(Solver):
    """Multigrid-preconditioned CG (reference _solvers.py:330-660)."""

    _COARSE = ("cg", "gmres", "splu", "spsolve", "cholmod")

    def __init__(self, mesh, kernel, maxiter=1000, tol=1e-5, n_smooth=3, omega=0.5, n_level=3, cycle="W",
                 w_level=1, coarse_solver="cholmod", matrix_free=False, low_level_tol=1e-8,
                 low_level_maxiter=5000, min_omega=0.4, omega_boost=1.06, *, precision="fp64", check_every=4,
                 warm_start=None, coarse_op="auto", coarse_correction=None, fixed_omega=None):
        self.kernel = kernel
        self.warm_start = warm_start
        self.coarse_correction = coarse_correction
        self.mesh = mesh
        self.last_x0 = None
        self.tol = tol
        self.maxiter = maxiter
        self.n_smooth = n_smooth
        self.omega = omega
        self.max_omega = omega
        self.min_omega = max(omega / 2, min_omega)
        self.d_omega = self.max_omega - self.min_omega
        self.omega_boost = omega_boost
        self.n_level = n_level
        self.cycle = cycle
        self.w_level = [w_level] if isinstance(w_level, int) else list(w_level)
        self.matrix_free = matrix_free
        self.dof = mesh.dof
        self.coarse_solver = coarse_solver
        self.low_level_tol = low_level_tol
        self.low_level_maxiter = low_level_maxiter
        self.precision = precision
        self.check_every = check_every
        if coarse_solver in ("splu", "spsolve") and matrix_free:
            raise ValueError("Matrix free is not supported with splu solver use cg instead.")
        if coarse_solver not in self._COARSE:
            raise ValueError("Coarse solver not recognized.")
        if matrix_free:
            raise NotImplementedError("Matrix free is not implemented yet.")
        # the reference takes its second coarse correction only for a lower-case 'w'
        # (_solvers.py:550); any other cycle name runs V-cycles
        if cycle == "w" and any(not (0 <= int(l) < 32) for l in self.w_level):
            raise ValueError("w_level entries must be levels 0..31")
        if precision not in ("fp64", "mixed", "mixed_bf16"):
            raise ValueError("precision must be 'fp64', 'mixed' or 'mixed_bf16'")
        if coarse_op not in ("auto", "element", "stencil"):
            raise ValueError("coarse_op must be 'auto', 'element' or 'stencil'")
        self.coarse_op = coarse_op
        if fixed_omega is not None and not (0.0 < float(fixed_omega) < 2.0):
            raise ValueError("fixed_omega must be a Jacobi weight in (0, 2) or None")
        self.fixed_omega = None if fixed_omega is None else float(fixed_omega)
        self._min_omega_arg = min_omega
        self._mg = None
        self._side = None
        self.last_info = None

    def _ensure(self):
        if self._mg is not None:
            return
        cfg = _lib.pf_mg_config()
        cfg.n_level = int(self.n_level)
        cfg.n_smooth = int(self.n_smooth)
        cfg.omega = float(self.omega)
        cfg.min_omega = float(self._min_omega_arg)
        cfg.omega_boost = float(self.omega_boost)
        cfg.coarse_beta = 1e-6
        cfg.precision = {"fp64": 0, "mixed": 1, "mixed_bf16": 2}[self.precision]
        cfg.check_every = int(self.check_every)
        element = self.coarse_op == "element" or (self.coarse_op == "auto" and self.precision != "fp64")
        cfg.coarse_op = 0 if element else 1
        cfg.w_mask = sum(1 << int(l) for l in set(self.w_level)) if self.cycle == "w" else 0
        cfg.omega_fixed = 0.0 if self.fixed_omega is None else self.fixed_omega
        h = ctypes.c_void_p()
        _lib.check(_lib.load().pf_mg_create(self.kernel._op, ctypes.byref(cfg), ctypes.byref(h)))
        self._mg = h

    def __del__(self):
        h = getattr(self, "_mg", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.pf_mg_destroy(h)
            self._mg = None

    def reset(self):
        """Drop the cached hierarchy (rebuilt on the next solve)."""
        if self._mg is not None:
            _lib.load().pf_mg_destroy(self._mg)
            self._mg = None

    def setup(self):
        """Build the hierarchy for the kernel's current rho and constraints."""
        self._ensure()
        k = self.kernel
        _lib.check(_lib.load().pf_mg_setup(self._mg, _lib.ptr(k.rho), k._mask_ptr(), _lib.stream()))

    def vcycle(self, r, omega=None):
        """One V-cycle from a zero guess (reference _multi_grid(0, r, 0)); needs setup()."""
        r = as_cuda(r, torch.float64)
        z = torch.empty_like(r)
        w = self.min_omega if omega is None else float(omega)
        _lib.check(_lib.load().pf_mg_vcycle(self._mg, _lib.ptr(r), _lib.ptr(z), w, _lib.stream()))
        return z

    def level_matvec(self, level, u):
        """y = A_level u with the operator the V-cycle applies on that level (needs setup());
        float64 for precision 'fp64', float32 otherwise."""
        dt = torch.float64 if self.precision == "fp64" else torch.float32
        u = as_cuda(u, dt)
        y = torch.empty_like(u)
        _lib.check(_lib.load().pf_mg_level_matvec(self._mg, int(level), _lib.ptr(u), _lib.ptr(y), _lib.stream()))
        return y

    def level_info(self):
        """(level 1 applied element by element, number of its coarse elements with an
        explicit matrix) of the current hierarchy."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.load().pf_mg_level_info(self._mg, ctypes.byref(a), ctypes.byref(b)))
        return bool(a.value), int(b.value)

    def solve(self, rhs, rho=None, use_last=True):
        k = self.kernel
        if not (k.has_rho or rho is not None):
            raise ValueError("Solver requires a density vector to be passed or set on the kernel.")
        if rho is not None:
            k.set_rho(rho)
        rhs = as_cuda(rhs, torch.float64)
        n = rhs.shape[0]
        warm = use_last and self.last_x0 is not None
        if warm and self.warm_start is not None and getattr(self.warm_start, "with_previous", False):
            x = self.warm_start.guess(k, rhs, prev=self.last_x0).clone()
        elif warm:
            x = self.last_x0
        elif self.warm_start is not None:
            x = self.warm_start.guess(k, rhs).clone()
            warm = True
        else:
            x = torch.empty(n, dtype=torch.float64, device=device())
        y = None
        if self.coarse_correction is not None:
            # the network runs on a side stream while the hierarchy is built on this one: it
            # needs only rho, the load and the constraints
            main = torch.cuda.current_stream()
            if self._side is None:
                self._side = torch.cuda.Stream()
            self._side.wait_stream(main)
            with torch.cuda.stream(self._side):
                y = as_cuda(self.coarse_correction.field(k, rhs), torch.float64)
        self.setup()
        if y is not None:
            main.wait_stream(self._side)
            _lib.check(_lib.load().pf_mg_set_deflation(self._mg, _lib.ptr(y), _lib.stream()))
        info = _lib.pf_solve_info()
        _lib.check(_lib.load().pf_mg_solve(self._mg, _lib.ptr(rhs), _lib.ptr(x), int(warm), float(self.tol),
                                           int(self.maxiter), ctypes.byref(info), _lib.stream()))
        self.last_info = _info(info)
        self.last_x0 = x
        return x, float(info.residual)
