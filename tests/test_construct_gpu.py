"""GPU: explicit CSR assembly (StructuredStiffnessKernel.construct, reference
stiffness/CUDA/_FEA.py:484-516) against the oracle.

The CSR must be the matrix the matvec applies, Z K Z + (I - Z): its dense form times
every unit vector equals the oracle's matvec (1e-13 relative, max-norm), it is symmetric,
its columns increase within each row, and its pattern has the closed-form count
dof^2 prod(3 nn_a - 2)."""
import numpy as np
import pytest
import torch

from conftest import rel, unit_K0
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _kernel(nel, cons):
    from pyfantom_b200.CUDA import StructuredMesh2D, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    phys = LinearElasticity(E=1.0, nu=0.3)
    mesh = StructuredMesh3D(*nel, *nel, physics=phys) if len(nel) == 3 else StructuredMesh2D(*nel, *nel, physics=phys)
    kern = StructuredStiffnessKernel(mesh)
    if len(cons):
        kern.add_constraints(torch.as_tensor(cons, device="cuda"))
    return kern


@pytest.mark.parametrize("nel", [(5, 4, 3), (2, 2, 7), (1, 1, 1), (7, 5), (1, 3), (12, 2)])
@pytest.mark.parametrize("constrained", [False, True])
def test_construct_equals_matvec_operator(nel, constrained):
    dim = len(nel)
    rng = np.random.default_rng(sum(nel) + 7 * constrained)
    n = int(np.prod(np.array(nel) + 1)) * dim
    cons = np.unique(rng.choice(n, size=max(1, n // 7), replace=False)) if constrained else np.array([], dtype=np.int64)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    kern = _kernel(nel, cons)
    Et = torch.as_tensor(E, device="cuda")
    csr = kern.construct(Et)
    nn = np.array(nel) + 1
    assert csr._nnz() == dim * dim * int(np.prod(3 * nn - 2))
    crow, col = csr.crow_indices().cpu().numpy(), csr.col_indices().cpu().numpy()
    for r in range(n):
        c = col[crow[r]:crow[r + 1]]
        assert np.all(np.diff(c) > 0)
    dense = csr.to_dense().cpu().numpy()
    ref = np.stack([O.matvec(nel, unit_K0(dim), E, np.eye(n)[:, j], cons if constrained else None) for j in range(n)], 1)
    assert rel(dense, ref) < 1e-13
    assert rel(dense, dense.T) < 1e-14
    # the second call reuses the pattern and follows new densities
    E2 = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    csr2 = kern.construct(torch.as_tensor(E2, device="cuda"))
    u = rng.standard_normal(n)
    y = (csr2 @ torch.as_tensor(u, device="cuda").unsqueeze(1)).squeeze(1).cpu().numpy()
    assert rel(y, O.matvec(nel, unit_K0(dim), E2, u, cons if constrained else None)) < 1e-13
