"""Structured meshes and density filters (drop-in for pyFANTOM/geom/CUDA and geom/commons).

* ``CuStructuredMesh2D/3D`` mirror pyFANTOM/geom/CUDA/_mesh.py:11-170: the same attributes
  (``nelx.., nel, dim, elements, nodes, elements_size, dx.., K_single, locals, A_single,
  As, volume, dof, dtype, physics, centroids``).  ``elements``, ``nodes`` and
  ``centroids`` are built on first access (the solver never needs them: the mesh is
  structured), as CUDA tensors in the reference orderings.
* ``CuStructuredFilter2D/3D`` mirror pyFANTOM/geom/CUDA/_filters.py:14-201 with the base
  class of pyFANTOM/geom/commons/_filters.py:19-156 (``dot``, ``_matvec``, ``_rmatvec``,
  ``T``, ``@``).  Forward and adjoint run in the library's filter kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._tensor import as_cuda, device
from .physics import LinearElasticity, Physx

__all__ = ["Mesh", "StructuredMesh", "CuStructuredMesh2D", "CuStructuredMesh3D", "FilterKernel",
           "CuStructuredFilter2D", "CuStructuredFilter3D"]


class Mesh:
    """Mesh base (pyFANTOM/geom/commons/_mesh.py)."""


class StructuredMesh(Mesh):
    """Structured mesh base (pyFANTOM/geom/commons/_mesh.py)."""


def _unit_element(h):
    h = np.asarray(h, dtype=np.float64)
    if h.size == 3:
        s = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    else:
        s = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    return s * h


class _StructuredMeshBase(StructuredMesh):
    def _common(self, nel, lengths, dtype, physics: Physx):
        self.nel = np.array(nel, dtype=np.int32)
        self.dim = np.array(lengths, dtype=dtype)
        h = tuple(float(lengths[a]) / int(nel[a]) for a in range(len(nel)))
        single = _unit_element(h)
        K = np.asarray(physics.K(single), dtype=np.float64)
        self.K_single_host = K
        self.elements_size = single.shape[0]
        self.dof = int(K.shape[0] / self.elements_size)
        self.dtype = dtype
        self.physics = physics
        self.K_single = torch.as_tensor(K, dtype=torch.float64, device=device())
        self.locals = [torch.as_tensor(np.asarray(a), dtype=torch.float64, device=device())
                       for a in physics.locals(single)]
        A = float(np.prod(h))
        self.A_single = torch.tensor([A], dtype=torch.float64, device=device())
        self.As = self.A_single
        self.volume = self.A_single[0] * int(np.prod(self.nel))
        self.n_nodes = int(np.prod(self.nel + 1))
        self._elements = None
        self._nodes = None
        self._centroids = None

    @property
    def elements(self):
        if self._elements is None:
            self._elements = _structured_elements(self.nel)
        return self._elements

    @property
    def nodes(self):
        if self._nodes is None:
            self._nodes = _structured_nodes(self.nel, self.dim)
        return self._nodes

    @property
    def centroids(self):
        if self._centroids is None:
            nel, L = self.nel, np.asarray(self.dim, dtype=np.float64)
            axes = [torch.linspace(L[a] / nel[a] / 2, L[a] - L[a] / nel[a] / 2, int(nel[a]),
                                   dtype=torch.float64, device=device()) for a in range(len(nel))]
            grids = torch.meshgrid(*axes, indexing="ij")
            self._centroids = torch.stack(grids, dim=-1).reshape(-1, len(nel))
        return self._centroids


def _structured_elements(nel):
    """Element connectivity in the reference order (core/CUDA/Kernels/_geom.py:3-49)."""
    dev = device()
    if len(nel) == 3:
        NX, NY, NZ = (int(v) for v in nel)
        nx, nz = NX + 1, NZ + 1
        i = torch.arange(NX, device=dev).view(-1, 1, 1)
        j = torch.arange(NY, device=dev).view(1, -1, 1)
        k = torch.arange(NZ, device=dev).view(1, 1, -1)
        base = (k + nz * i + nz * nx * j).reshape(-1)
        off = torch.tensor([0, nz, nz + nz * nx, nz * nx, 1, nz + 1, nz + nz * nx + 1, nz * nx + 1], device=dev)
        return (base[:, None] + off[None, :]).to(torch.int32)
    NX, NY = (int(v) for v in nel)
    nx = NX + 1
    i = torch.arange(NX, device=dev).view(-1, 1)
    j = torch.arange(NY, device=dev).view(1, -1)
    base = (j * nx + i).reshape(-1)
    off = torch.tensor([0, 1, nx + 1, nx], device=dev)
    return (base[:, None] + off[None, :]).to(torch.int32)


def _structured_nodes(nel, lengths):
    """Node coordinates in the reference order (meshgrid(x, y[, z]) default indexing)."""
    dev = device()
    axes = [torch.linspace(0, float(lengths[a]), int(nel[a]) + 1, dtype=torch.float64, device=dev)
            for a in range(len(nel))]
    grids = torch.meshgrid(*axes, indexing="xy")
    return torch.stack([g.reshape(-1) for g in grids], dim=-1)


class CuStructuredMesh2D(_StructuredMeshBase):
    """2D structured Q4 mesh (pyFANTOM/geom/CUDA/_mesh.py:11-86)."""

    def __init__(self, nx, ny, lx, ly, dtype=np.float64, physics: Physx = LinearElasticity(E=1.0, nu=1 / 3)):
        self.nelx, self.nely = int(nx), int(ny)
        self.lx, self.ly = lx, ly
        self.dx, self.dy = lx / nx, ly / ny
        self._common((nx, ny), (lx, ly), dtype, physics)


class CuStructuredMesh3D(_StructuredMeshBase):
    """3D structured H8 mesh (pyFANTOM/geom/CUDA/_mesh.py:89-170)."""

    def __init__(self, nx, ny, nz, lx, ly, lz, dtype=np.float64, physics: Physx = LinearElasticity(E=1.0, nu=1 / 3)):
        self.nelx, self.nely, self.nelz = int(nx), int(ny), int(nz)
        self.lx, self.ly, self.lz = lx, ly, lz
        self.dx, self.dy, self.dz = lx / nx, ly / ny, lz / nz
        self._common((nx, ny, nz), (lx, ly, lz), dtype, physics)


# -----------------------------------------------------------------------------------------
# filters
# -----------------------------------------------------------------------------------------
class _TransposeView:
    def __init__(self, original):
        self._original = original

    def __matmul__(self, rhs):
        return self._original._rmatvec(rhs)

    def dot(self, rhs):
        return self._original._rmatvec(rhs)

    @property
    def T(self):
        return self._original


class FilterKernel:
    """Filter base (pyFANTOM/geom/commons/_filters.py:19-156)."""

    def __init__(self):
        self.weights = None
        self.offsets = None
        self.shape = None
        self.matvec = self.dot

    def _matvec(self, rho):
        raise NotImplementedError("_matvec method must be implemented in subclasses.")

    def _rmatvec(self, rho):
        raise NotImplementedError("_rmatvec method must be implemented in subclasses.")

    def dot(self, rho):
        if isinstance(rho, torch.Tensor) and rho.is_cuda:
            if rho.ndim == 1:
                if rho.shape[0] == self.shape[1]:
                    return self._matvec(rho)
                raise ValueError("Input vector size does not match the filter kernel size.")
            raise NotImplementedError("Only vector inputs are supported.")
        raise ValueError("Input must be a CUDA torch.Tensor vector.")

    def __matmul__(self, rhs):
        return self.dot(rhs)

    @property
    def T(self):
        return _TransposeView(self)


def cone_weights(nel, h, r_min):
    """Cone weights and offsets (pyFANTOM/geom/CUDA/_filters.py:65-98): offsets over
    [-ceil(r), ceil(r)]^dim in meshgrid 'ij' order, distance scaled by h / min(h),
    w = (r - d) / r kept where positive, normalised to sum 1."""
    dim = len(nel)
    scales = np.asarray(h, dtype=np.float64)
    scales = scales / scales.min()
    n = int(np.ceil(r_min))
    rng = np.arange(-n, n + 1, dtype=np.int32)
    grids = np.meshgrid(*([rng] * dim), indexing="ij")
    offsets = np.vstack([g.ravel() for g in grids]).T
    d = np.linalg.norm(offsets * scales[None], axis=1)
    w = (r_min - d) / r_min
    keep = w > 0
    offsets, w = offsets[keep], w[keep]
    w = w / w.sum()
    return w.astype(np.float64), np.ascontiguousarray(offsets.astype(np.int32))


class _StructuredFilter(FilterKernel):
    def _setup(self, mesh, r_min, h):
        super().__init__()
        _lib.require_cuda()
        lib = _lib.load()
        self.r_min = r_min
        self.dtype = mesh.dtype
        n = int(np.prod(self._nel))
        self.shape = (n, n)
        w, off = cone_weights(self._nel, h, r_min)
        self._grid = _lib.make_grid(self._nel)
        handle = ctypes.c_void_p()
        _lib.check(lib.pf_filter_create(ctypes.byref(self._grid), len(w), off.ctypes.data, w.ctypes.data,
                                        ctypes.byref(handle)))
        self._handle = handle
        self.weights = torch.as_tensor(w, device=device())
        self.offsets = torch.as_tensor(off, device=device())
        self.normalizer = torch.empty(n, dtype=torch.float64, device=device())
        _lib.check(lib.pf_filter_normalizer_f64(self._handle, _lib.ptr(self.normalizer), _lib.stream()))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.pf_filter_destroy(h)
            self._handle = None

    def _matvec(self, rho):
        rho = as_cuda(rho, torch.float64)
        out = torch.empty_like(rho)
        _lib.check(_lib.load().pf_filter_fwd_f64(self._handle, _lib.ptr(rho), _lib.ptr(out), _lib.stream()))
        return out

    def _rmatvec(self, rho):
        rho = as_cuda(rho, torch.float64)
        out = torch.empty_like(rho)
        _lib.check(_lib.load().pf_filter_adj_f64(self._handle, _lib.ptr(rho), _lib.ptr(out), _lib.stream()))
        return out


class CuStructuredFilter3D(_StructuredFilter):
    """3D cone filter (pyFANTOM/geom/CUDA/_filters.py:14-108)."""

    def __init__(self, mesh: CuStructuredMesh3D, r_min):
        self.nelx, self.nely, self.nelz = (int(v) for v in mesh.nel)
        self._nel = (self.nelx, self.nely, self.nelz)
        self._setup(mesh, r_min, (mesh.dx, mesh.dy, mesh.dz))


class CuStructuredFilter2D(_StructuredFilter):
    """2D cone filter (pyFANTOM/geom/CUDA/_filters.py:111-201)."""

    def __init__(self, mesh: CuStructuredMesh2D, r_min):
        self.nelx, self.nely = (int(v) for v in mesh.nel)
        self._nel = (self.nelx, self.nely)
        self._setup(mesh, r_min, (mesh.dx, mesh.dy))
