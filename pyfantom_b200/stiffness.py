"""Structured stiffness operator (drop-in for pyFANTOM/stiffness/CUDA/_FEA.py:6-673).

``StructuredStiffnessKernel`` keeps the reference object API: ``set_rho``, ``dot`` /
``matvec`` / ``rmatvec`` / ``@``, ``diagonal(rho=None)``, ``set_constraints``,
``add_constraints``, ``process_grad``, ``reset`` and the attributes ``shape, dtype,
constraints, has_con (alias has_cons), rho, has_rho, non_con_map, K_single, n_nodes,
dof, elements_size, mat_vec, diag, dk``.  As in the reference, ``dot`` writes into the
persistent buffer ``mat_vec`` and returns it (the next call overwrites it), ``set_rho``
keeps a reference to the given (already penalised) densities, and Dirichlet DOFs act as
identity rows and skipped columns.

The matrix-free product, diagonal and element sensitivity run in the library kernels
(``pf_matvec_f64``, ``pf_diagonal_f64``, ``pf_sensitivity_f64``).  The explicit CSR
assembly of ``construct`` (used by the reference's direct solvers) is outside this
build and raises ``NotImplementedError``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._tensor import as_cuda, device

__all__ = ["StiffnessKernel", "StructuredStiffnessKernel"]


class StiffnessKernel:
    """Stiffness kernel base (pyFANTOM/stiffness/CUDA/_FEA.py:6-262)."""

    def __init__(self):
        self.has_rho = False
        self.rho = None
        self.shape = None
        self.matvec = self.dot
        self.rmatvec = self.dot
        self.matmat = self.dot
        self.rmatmat = self.dot
        self.mat_vec = None
        self.diag = None
        self.dk = None

    def set_rho(self, rho):
        self.rho = as_cuda(rho, torch.float64)
        self.has_rho = True

    def dot(self, rhs):
        raise NotImplementedError

    def __matmul__(self, rhs):
        return self.dot(rhs)


class StructuredStiffnessKernel(StiffnessKernel):
    """Matrix-free K(rho) on a structured Q4/H8 mesh (reference _FEA.py:265-673)."""

    def __init__(self, mesh):
        super().__init__()
        _lib.require_cuda()
        lib = _lib.load()
        self.mesh = mesh
        self.dof = mesh.dof
        self.K_single = mesh.K_single
        self.dtype = mesh.dtype
        self.elements_size = mesh.elements_size
        self.n_nodes = int(np.prod(np.asarray(mesh.nel) + 1))
        self.nel = tuple(int(v) for v in mesh.nel)
        n = self.n_nodes * self.dof
        self.shape = (n, n)
        self.constraints = torch.zeros(n, dtype=torch.bool, device=device())
        self.node_mask = torch.zeros(self.n_nodes, dtype=torch.uint8, device=device())
        self.has_con = False
        self.idx_map = torch.arange(n, dtype=torch.int32, device=device())
        self.non_con_map = self.idx_map
        self.has_been_constructed = False
        self._csr_vals = None
        self.ptr = None
        self._grid = _lib.make_grid(self.nel)
        handle = ctypes.c_void_p()
        K0 = np.ascontiguousarray(mesh.K_single_host, dtype=np.float64)
        _lib.check(lib.pf_op_create(ctypes.byref(self._grid), K0.ctypes.data, ctypes.byref(handle)))
        self._op = handle

    def __del__(self):
        h = getattr(self, "_op", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.pf_op_destroy(h)
            self._op = None

    # --- reference attribute aliases ---------------------------------------------------
    @property
    def has_cons(self):
        return self.has_con

    @has_cons.setter
    def has_cons(self, v):
        self.has_con = bool(v)

    @property
    def nodes(self):
        return self.mesh.nodes

    @property
    def elements(self):
        return self.mesh.elements

    @property
    def elements_flat(self):
        return self.mesh.elements.reshape(-1)

    @property
    def el_ids(self):
        return torch.arange(self.mesh.elements.shape[0], dtype=torch.int32, device=device()).repeat_interleave(
            self.elements_size)

    @property
    def sorter(self):
        return torch.argsort(self.elements_flat, stable=True).to(torch.int32)

    @property
    def node_ids(self):
        ef = self.elements_flat.to(torch.int64)
        return torch.searchsorted(ef[self.sorter.to(torch.int64)],
                                  torch.arange(self.n_nodes, device=device())).to(torch.int32)

    # --- constraints -------------------------------------------------------------------
    def _refresh_mask(self):
        _lib.check(_lib.load().pf_pack_mask(self._op, _lib.ptr(self.constraints.view(torch.uint8)),
                                            _lib.ptr(self.node_mask), _lib.stream()))
        self.non_con_map = self.idx_map[~self.constraints]

    def set_constraints(self, constraints):
        self.constraints[:] = False
        idx = as_cuda(constraints, torch.int64) if len(constraints) else None
        if idx is not None:
            self.constraints[idx] = True
        self.has_con = True
        self._refresh_mask()

    def add_constraints(self, constraints):
        idx = as_cuda(constraints, torch.int64)
        if idx.numel():
            self.constraints[idx] = True
        self.has_con = True
        self._refresh_mask()

    def _mask_ptr(self):
        return _lib.ptr(self.node_mask) if self.has_con else _lib.ptr(None)

    # --- operator ----------------------------------------------------------------------
    def _matvec(self, rho, vec):
        vec = as_cuda(vec, torch.float64)
        if self.mat_vec is None or self.mat_vec.shape[0] != self.shape[0]:
            self.mat_vec = torch.empty(self.shape[0], dtype=torch.float64, device=device())
        if vec.data_ptr() == self.mat_vec.data_ptr():
            vec = vec.clone()
        _lib.check(_lib.load().pf_matvec_f64(self._op, _lib.ptr(rho), _lib.ptr(vec), self._mask_ptr(),
                                             _lib.ptr(self.mat_vec), _lib.stream()))
        return self.mat_vec

    def _rmatvec(self, rho, vec):
        return self._matvec(rho, vec)

    def dot(self, rhs):
        if not self.has_rho:
            raise ValueError("Rho has not been set. dot works only after setting rho.")
        if isinstance(rhs, torch.Tensor):
            if rhs.shape[0] != self.shape[0]:
                raise ValueError("Shape of the input vector does not match the number of nodes and dof.")
            if rhs.ndim == 1:
                return self._matvec(self.rho, rhs)
            if rhs.ndim == 2:  # column-by-column product for dense multi-vectors
                return torch.stack([self._matvec(self.rho, rhs[:, c]).clone() for c in range(rhs.shape[1])], dim=1)
        raise NotImplementedError("Only CUDA torch tensors (vectors or dense matrices) are supported.")

    def diagonal(self, rho=None):
        if rho is None and not self.has_rho:
            raise ValueError("Rho has not been set. diagonal works only after setting rho or if rho is provided.")
        r = self.rho if rho is None else as_cuda(rho, torch.float64)
        if self.diag is None:
            self.diag = torch.empty(self.shape[0], dtype=torch.float64, device=device())
        _lib.check(_lib.load().pf_diagonal_f64(self._op, _lib.ptr(r), self._mask_ptr(), _lib.ptr(self.diag),
                                               _lib.stream()))
        return self.diag

    def process_grad(self, U):
        U = as_cuda(U, torch.float64)
        n_el = int(np.prod(self.nel))
        if self.dk is None or self.dk.shape[0] != n_el:
            self.dk = torch.empty(n_el, dtype=torch.float64, device=device())
        _lib.check(_lib.load().pf_sensitivity_f64(self._op, _lib.ptr(U), _lib.ptr(self.dk), _lib.stream()))
        return self.dk

    def construct(self, rho):
        """Explicit sparse matrix on the GPU (reference _FEA.py:484-516): a torch CSR tensor
        (int32 indices, float64 values) of the matrix ``dot`` applies, Z K(rho) Z + (I - Z)
        with Z zeroing the constrained DOFs.  The sparsity pattern is kept across calls
        (``self.ptr``), as the reference keeps its ``indptr``."""
        L = _lib.load()
        rho = as_cuda(rho, torch.float64)
        n = self.shape[0]
        dev = device()
        if not self.has_been_constructed or self._csr_vals is None:
            nnz = int(L.pf_csr_nnz(self._op))
            self.ptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
            self._csr_cols = torch.empty(nnz, dtype=torch.int32, device=dev)
            self._csr_vals = torch.empty(nnz, dtype=torch.float64, device=dev)
        _lib.check(L.pf_construct_csr_f64(self._op, _lib.ptr(rho), self._mask_ptr(), _lib.ptr(self.ptr),
                                          _lib.ptr(self._csr_cols), _lib.ptr(self._csr_vals), _lib.stream()))
        self.CSR = torch.sparse_csr_tensor(self.ptr, self._csr_cols, self._csr_vals, size=(n, n))
        self.has_been_constructed = True
        return self.CSR

    def reset(self):
        self.has_rho = False
        self.rho = None
        self.has_been_constructed = False
        self._csr_vals = None
        self.constraints[:] = False
        self.node_mask.zero_()
        self.has_con = False
        self.non_con_map = self.idx_map
        self.mat_vec = None
        self.diag = None
        self.dk = None
