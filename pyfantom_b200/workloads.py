"""Synthetic SIMP workloads on structured meshes (host-side numpy builders).

Each builder returns plain numpy arrays describing one linear-elasticity problem on a
structured Q4/H8 mesh with unit elements (h = 1):

* ``fixed_dofs``  - int64 indices of Dirichlet DOFs (prescribed value 0);
* ``rhs``         - float64 load vector (DOF order ``node*dof + d``);
* ``x``           - float64 seeded, Gaussian-smoothed densities in element order;
* ``E``           - penalised stiffness ``clip(x**3, 1e-9, 1)`` (the SIMP law with
  ``void=1e-9, heavyside=False``, pyFANTOM/Problem/CUDA/MinimumCompliance.py:305-324).

Node and element orderings follow the reference structured mesh
(pyFANTOM/core/CUDA/Kernels/_geom.py:23-49,94-114): 3D node ``k + nz*i + nz*nx*j``
(z fastest, then x, then y), element ``i*nely*nelz + j*nelz + k``; 2D node ``i + nx*j``,
element ``i*nely + j``.

Boundary conditions and loads restate the reference documentation's conventions
(y vertical; docs/source/examples/3d_topology_optimization.rst:85-97):

* cantilever: all DOFs fixed on the face x == 0; unit downward load spread over the
  nodes of the edge (x == nelx, y == 0);
* bridge: all DOFs fixed on the lines (x == 0, y == 0) and (x == nelx, y == 0); unit
  downward load spread over the top face y == nely;
* MBB half-beam (2D): x-roller on the left edge, y-roller at the bottom-right node,
  unit downward point load at the top-left node.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "node_index_3d", "node_index_2d", "cantilever3d", "bridge3d", "mbb2d",
    "smoothed_density", "simp_E",
]


def node_index_3d(i, j, k, nelx, nely, nelz):
    """Reference 3D node index for node coordinates (i, j, k) (x, y, z)."""
    nx, nz = nelx + 1, nelz + 1
    return np.asarray(k) + nz * np.asarray(i) + nz * nx * np.asarray(j)


def node_index_2d(i, j, nelx, nely):
    """Reference 2D node index for node coordinates (i, j) (x, y)."""
    return np.asarray(i) + (nelx + 1) * np.asarray(j)


def smoothed_density(shape, seed: int, sigma: float = 2.0, lo: float = 0.001, hi: float = 1.0):
    """uniform(lo, hi) field of ``shape`` from ``default_rng(seed)``, Gaussian-smoothed with
    ``sigma`` (scipy ``reflect`` mode), flattened in C order (= reference element order)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo, hi, size=shape)
    return gaussian_filter(x, sigma=sigma).reshape(-1).astype(np.float64)


def simp_E(x, penalty: float = 3.0, void: float = 1e-9):
    """E = clip(clip(x**p, void, 1) * 1.0, void, inf) (single material, no projection)."""
    e = np.clip(np.asarray(x, dtype=np.float64) ** penalty, void, 1.0)
    return np.clip(e, void, None)


def _dofs_of(nodes, dof):
    nodes = np.asarray(nodes, dtype=np.int64).reshape(-1)
    return (nodes[:, None] * dof + np.arange(dof)[None, :]).reshape(-1)


def cantilever3d(nelx: int, nely: int, nelz: int, seed: int = 0):
    """Cantilever on a (nelx, nely, nelz) H8 mesh (see module docstring)."""
    n_nodes = (nelx + 1) * (nely + 1) * (nelz + 1)
    J, K = np.meshgrid(np.arange(nely + 1), np.arange(nelz + 1), indexing="ij")
    fixed_nodes = np.sort(node_index_3d(np.zeros_like(J), J, K, nelx, nely, nelz).reshape(-1))
    ks = np.arange(nelz + 1)
    load_nodes = node_index_3d(np.full_like(ks, nelx), np.zeros_like(ks), ks, nelx, nely, nelz)
    rhs = np.zeros(n_nodes * 3)
    rhs[load_nodes * 3 + 1] = -1.0 / len(load_nodes)
    x = smoothed_density((nelx, nely, nelz), seed)
    return dict(nel=(nelx, nely, nelz), dim=3, dof=3, n_nodes=n_nodes,
                fixed_dofs=_dofs_of(fixed_nodes, 3), rhs=rhs, x=x, E=simp_E(x),
                fixed_nodes=fixed_nodes, load_nodes=load_nodes,
                load_forces=np.tile([0.0, -1.0 / len(load_nodes), 0.0], (len(load_nodes), 1)))


def bridge3d(nelx: int, nely: int, nelz: int, seed: int = 0):
    """Bridge on a (nelx, nely, nelz) H8 mesh (see module docstring)."""
    n_nodes = (nelx + 1) * (nely + 1) * (nelz + 1)
    ks = np.arange(nelz + 1)
    left = node_index_3d(np.zeros_like(ks), np.zeros_like(ks), ks, nelx, nely, nelz)
    right = node_index_3d(np.full_like(ks, nelx), np.zeros_like(ks), ks, nelx, nely, nelz)
    fixed_nodes = np.sort(np.concatenate([left, right]))
    I, K = np.meshgrid(np.arange(nelx + 1), np.arange(nelz + 1), indexing="ij")
    top = np.sort(node_index_3d(I, np.full_like(I, nely), K, nelx, nely, nelz).reshape(-1))
    rhs = np.zeros(n_nodes * 3)
    rhs[top * 3 + 1] = -1.0 / len(top)
    x = smoothed_density((nelx, nely, nelz), seed)
    return dict(nel=(nelx, nely, nelz), dim=3, dof=3, n_nodes=n_nodes,
                fixed_dofs=_dofs_of(fixed_nodes, 3), rhs=rhs, x=x, E=simp_E(x),
                fixed_nodes=fixed_nodes, load_nodes=top,
                load_forces=np.tile([0.0, -1.0 / len(top), 0.0], (len(top), 1)))


def mbb2d(nelx: int = 120, nely: int = 40):
    """MBB half-beam on a (nelx, nely) Q4 mesh (see module docstring)."""
    n_nodes = (nelx + 1) * (nely + 1)
    js = np.arange(nely + 1)
    left = node_index_2d(np.zeros_like(js), js, nelx, nely)
    br = int(node_index_2d(nelx, 0, nelx, nely))
    tl = int(node_index_2d(0, nely, nelx, nely))
    fixed = np.sort(np.concatenate([left * 2 + 0, [br * 2 + 1]]))
    rhs = np.zeros(n_nodes * 2)
    rhs[tl * 2 + 1] = -1.0
    x = np.full(nelx * nely, 0.5)
    return dict(nel=(nelx, nely), dim=2, dof=2, n_nodes=n_nodes, fixed_dofs=fixed.astype(np.int64),
                rhs=rhs, x=x, E=simp_E(x), left_nodes=left, br_node=br, tl_node=tl)
