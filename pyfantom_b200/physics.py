"""Element physics on the host: isotropic linear elasticity for Q4 and H8 elements.

The element stiffness matrix K0 is formed once per mesh on the host, exactly as the
reference forms it (pyFANTOM/physics/LinearElasticity.py:305-443 for Q4 with plane
stress / plane strain, :700-833 for H8): full Gauss quadrature (2x2 / 2x2x2), isotropic
constitutive matrix, ``K = sum_q w_q detJ B^T C B`` (times the thickness in 2D).  The DOF
order within an element is (node, component) and the local node order is the reference's
counter-clockwise order (bottom face first in 3D).
"""
from __future__ import annotations

import numpy as np

__all__ = ["Physx", "LinearElasticity"]

# quadrature abscissae exactly as written in the reference (Q4 uses a 15-digit literal)
_GP_Q4 = np.array([-0.577350269189626, 0.577350269189626])
_GP_H8 = np.array([-1.0 / np.sqrt(3.0), 1.0 / np.sqrt(3.0)])
# local node signs (xi, eta[, zeta]) of the reference element node order
_Q4_SIGNS = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], dtype=np.float64)
_H8_SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


class Physx:
    """Physics interface (pyFANTOM/physics/_physx.py:1-45)."""

    def K(self, x0s):
        raise NotImplementedError("K method must be implemented in subclasses.")

    def locals(self, x0s):
        raise NotImplementedError("locals method must be implemented in subclasses.")

    def volume(self, x0s):
        raise NotImplementedError("volume method must be implemented in subclasses.")

    def neumann(self, x0s):
        raise NotImplementedError("neumann method must be implemented in subclasses.")


def _c_matrix_3d(E, nu):
    f = E / ((1 + nu) * (1 - 2 * nu))
    C = np.zeros((6, 6))
    C[:3, :3] = f * nu
    np.fill_diagonal(C[:3, :3], f * (1 - nu))
    C[3, 3] = C[4, 4] = C[5, 5] = f * (1 - 2 * nu) / 2
    return C


def _d_matrix_2d(E, nu, plane_strain):
    D = np.zeros((3, 3))
    if not plane_strain:
        c = E / (1 - nu * nu)
        D[0, 0] = D[1, 1] = c
        D[0, 1] = D[1, 0] = c * nu
        D[2, 2] = c * (1 - nu) / 2
    else:
        c = E / ((1 + nu) * (1 - 2 * nu))
        D[0, 0] = D[1, 1] = c * (1 - nu)
        D[0, 1] = D[1, 0] = c * nu
        D[2, 2] = c * (1 - 2 * nu) / 2
    return D


def _h8(x0, E, nu):
    """(K 24x24, C 6x6, B_avg 6x24) for one hexahedron with nodes x0 (8x3)."""
    C = _c_matrix_3d(E, nu)
    K = np.zeros((24, 24))
    B_avg = np.zeros((6, 24))
    for xi1 in _GP_H8:
        for xi2 in _GP_H8:
            for xi3 in _GP_H8:
                s = _H8_SIGNS
                # derivatives of N_l = (1 + s1 xi1)(1 + s2 xi2)(1 + s3 xi3) / 8
                dN = np.stack([s[:, 0] * (1 + s[:, 1] * xi2) * (1 + s[:, 2] * xi3),
                               s[:, 1] * (1 + s[:, 0] * xi1) * (1 + s[:, 2] * xi3),
                               s[:, 2] * (1 + s[:, 0] * xi1) * (1 + s[:, 1] * xi2)]) / 8.0
                J = dN @ x0
                detJ = np.linalg.det(J)
                G = np.linalg.inv(J) @ dN  # 3 x 8 physical derivatives
                B = np.zeros((6, 24))
                for a in range(3):
                    B[a, a::3] = G[a]
                B[3, 0::3], B[3, 1::3] = G[1], G[0]
                B[4, 2::3], B[4, 1::3] = G[1], G[2]
                B[5, 0::3], B[5, 2::3] = G[2], G[0]
                K += detJ * (B.T @ C @ B)
                B_avg += B / 8
    return K, C, B_avg


def _q4(x0, E, nu, plane_strain, t):
    D = _d_matrix_2d(E, nu, plane_strain)
    K = np.zeros((8, 8))
    B_avg = np.zeros((3, 8))
    for r in _GP_Q4:
        for s_ in _GP_Q4:
            s = _Q4_SIGNS
            dN = np.stack([s[:, 0] * (1 + s[:, 1] * s_), s[:, 1] * (1 + s[:, 0] * r)]) / 4.0
            J = dN @ x0
            detJ = np.linalg.det(J)
            G = np.linalg.inv(J) @ dN
            B = np.zeros((3, 8))
            B[0, 0::2] = G[0]
            B[1, 1::2] = G[1]
            B[2, 0::2], B[2, 1::2] = G[1], G[0]
            K += t * detJ * (B.T @ D @ B)
            B_avg += B / 4
    return K, D, B_avg


class LinearElasticity(Physx):
    """Isotropic linear elasticity (pyFANTOM/physics/LinearElasticity.py:4-122); Q4 and H8.

    ``K(x0s)`` accepts one element (``(4,2)`` or ``(8,3)`` node coordinates) or a batch
    (``(n,4,2)`` / ``(n,8,3)``) and returns the element stiffness matrix (or a batch).
    """

    def __init__(self, E=1.0, nu=1.0 / 3.0, thickness=1.0, type="PlaneStress"):
        self.E = E
        self.nu = nu
        self.thickness = thickness
        self.type = 0 if type == "PlaneStress" else 1

    def _dispatch(self, x0s):
        x0s = np.asarray(x0s, dtype=np.float64)
        single = x0s.ndim == 2
        batch = x0s[None] if single else x0s
        if batch.shape[1:] == (8, 3):
            res = [_h8(x, self.E, self.nu) for x in batch]
        elif batch.shape[1:] == (4, 2):
            res = [_q4(x, self.E, self.nu, self.type == 1, self.thickness) for x in batch]
        else:
            raise ValueError("Invalid input shape (only Q4 (4,2) and H8 (8,3) elements are supported)")
        out = [np.stack([r[i] for r in res]) for i in range(3)]
        return [o[0] for o in out] if single else out

    def K(self, x0s):
        return self._dispatch(x0s)[0]

    def locals(self, x0s):
        return list(self._dispatch(x0s)[1:])

    def volume(self, x0s):
        x0s = np.asarray(x0s, dtype=np.float64)
        ext = x0s.max(axis=-2) - x0s.min(axis=-2)
        return np.prod(ext, axis=-1)

    def neumann(self, x0s):
        pass
