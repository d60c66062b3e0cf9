"""Boundary conditions, loads and the FE solve (drop-in for
pyFANTOM/FiniteElement/CUDA/FiniteElement.py:15-436 and FiniteElement/FiniteElement.py).

Semantics follow the reference: Dirichlet DOFs are registered on the stiffness kernel
(identity rows) and their prescribed values kept in ``d_rhs`` (NaN elsewhere);
``add_point_forces`` accumulates into ``rhs`` and then overwrites the Dirichlet entries
of ``rhs`` with ``d_rhs``; ``solve(rho)`` sets the (penalised) densities on the kernel
and calls ``solver.solve(rhs, use_last=True)``.  Positions are matched to the nearest
mesh node with a KD-tree on the host, as in the reference.  Plotting helpers of the
reference are not part of this library.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from ._tensor import as_cuda, device

__all__ = ["FE", "FiniteElement"]


class FE:
    """FE base (pyFANTOM/FiniteElement/FiniteElement.py:4-70)."""


class FiniteElement(FE):
    def __init__(self, mesh, kernel, solver):
        self.mesh = mesh
        self.kernel = kernel
        self.solver = solver
        self.dtype = mesh.dtype
        n = kernel.shape[0]
        self.rhs = torch.zeros(n, dtype=torch.float64, device=device())
        self.d_rhs = torch.full((n,), float("nan"), dtype=torch.float64, device=device())
        self.KDTree = None
        self.nel = int(np.prod(mesh.nel))
        self.is_3D = len(mesh.nel) == 3
        self.dof = mesh.dof

    def _nearest(self, positions):
        if self.KDTree is None:
            from scipy.spatial import KDTree
            self.KDTree = KDTree(self.mesh.nodes.cpu().numpy())
        pos = positions.cpu().numpy() if isinstance(positions, torch.Tensor) else np.asarray(positions)
        _, ids = self.KDTree.query(pos)
        return np.asarray(ids)

    def add_dirichlet_boundary_condition(self, node_ids: Optional[np.ndarray] = None, positions=None, dofs=None,
                                         rhs=0.):
        if node_ids is None and positions is None:
            raise ValueError("Either node_ids or positions must be provided.")
        if node_ids is not None and positions is not None:
            raise ValueError("Only one of node_ids or positions should be provided.")
        if node_ids is None:
            return self.add_dirichlet_boundary_condition(node_ids=self._nearest(positions), dofs=dofs, rhs=rhs)
        node_ids = as_cuda(node_ids, torch.int64).reshape(-1)
        N_con = node_ids.shape[0]
        scalar = isinstance(rhs, (float, int))
        if not scalar:
            rhs = as_cuda(rhs, torch.float64)
            if rhs.shape[0] != N_con:
                raise ValueError("rhs must have the same length as node_ids or positions.")
        if dofs is None:
            sel = torch.ones((N_con, self.dof), dtype=torch.bool, device=device())
        else:
            dofs = as_cuda(dofs, torch.int64)
            if dofs.ndim == 1:
                dofs = dofs.reshape(1, -1)
            if dofs.shape[0] != N_con and dofs.shape[0] != 1:
                raise ValueError("dofs must have the same length as node_ids.")
            if dofs.shape[0] == 1:
                dofs = dofs.expand(N_con, -1)
            sel = dofs == 1
        for i in range(self.dof):
            cons = node_ids[sel[:, i]] * self.dof + i
            self.kernel.add_constraints(cons)
            if scalar:
                self.d_rhs[cons] = float(rhs) + torch.nan_to_num(self.d_rhs[cons], nan=0.0)
            else:
                self.d_rhs[cons] = rhs[sel[:, i], i]

    def add_neumann_boundary_condition(self, **kwargs):
        raise NotImplementedError("Neumann boundary conditions are not implemented in this version of FiniteElement.")

    def add_point_forces(self, forces, node_ids=None, positions=None):
        if node_ids is None and positions is None:
            raise ValueError("Either node_ids or positions must be provided.")
        if node_ids is not None and positions is not None:
            raise ValueError("Only one of node_ids or positions should be provided.")
        if node_ids is None:
            return self.add_point_forces(forces=forces, node_ids=self._nearest(positions))
        node_ids = as_cuda(node_ids, torch.int64).reshape(-1)
        forces = as_cuda(forces, torch.float64)
        if forces.ndim == 1:
            forces = forces.reshape(1, -1)
        if (forces.shape[0] != node_ids.shape[0] and forces.shape[0] != 1) or forces.shape[1] != self.dof:
            raise ValueError("forces must have shape (N_forces, mesh.dof).")
        if forces.shape[0] == 1:
            forces = forces.expand(node_ids.shape[0], -1)
        for i in range(self.dof):
            self.rhs.index_add_(0, node_ids * self.dof + i, forces[:, i].contiguous())
        dirichlet = ~torch.isnan(self.d_rhs)
        self.rhs[dirichlet] = self.d_rhs[dirichlet]

    def reset_forces(self):
        self.rhs[:] = 0

    def reset_dirichlet_boundary_conditions(self):
        self.kernel.set_constraints([])
        self.kernel.has_cons = False
        self.d_rhs[:] = float("nan")

    def visualize_problem(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of this library")

    visualize_density = visualize_problem
    visualize_field = visualize_problem

    def solve(self, rho=None):
        if rho is not None and rho.shape[0] != self.nel:
            raise ValueError("rho must have the same length as the number of elements in the mesh.")
        if rho is None:
            rho = torch.ones(self.nel, dtype=torch.float64, device=device())
        self.kernel.set_rho(rho)
        return self.solver.solve(self.rhs, use_last=True)
