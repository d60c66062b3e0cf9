"""GPU: the learned coarse-grid correction of the MGCG (deflated PCG, pf_mg_set_deflation)
against the oracle's deflated PCG on the same deflation field.

The deflation space is spanned by the components of one nodal field (zero on constrained
DOFs); the solver starts from x0 = x + Q G^-1 Q^T (b - K x) and keeps its search directions
K-orthogonal to Q.  Parity bar: the FP64 form takes the oracle's iteration count (+-1) and
both reach the plain solve's solution (1e-8 relative, max-norm); the FP32 V-cycle form
(precision 'mixed') reaches the same solution within +-2 iterations of the oracle.  The
library rounds the field to FP32 (the basis Q) and keeps K Q in FP64; the oracle keeps both
in FP64.
"""
import numpy as np
import pytest
import torch

from conftest import rel, unit_K0
from oracle import oracle as O
from pyfantom_b200 import workloads

pytestmark = pytest.mark.gpu


class _Given:
    """coarse_correction that hands the solver a fixed nodal field."""

    def __init__(self, y):
        self.y = torch.as_tensor(np.ascontiguousarray(y), dtype=torch.float64, device="cuda")
        self.calls = 0

    def field(self, kern, rhs):
        self.calls += 1
        return self.y


def _problem(wl, n_level, precision, cc, tol=1e-10):
    from pyfantom_b200.CUDA import FiniteElement, MultiGrid, StructuredMesh2D, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    nel = wl["nel"]
    phys = LinearElasticity(E=1.0, nu=0.3)
    mesh = StructuredMesh3D(*nel, *nel, physics=phys) if len(nel) == 3 else StructuredMesh2D(*nel, *nel, physics=phys)
    kern = StructuredStiffnessKernel(mesh)
    sol = MultiGrid(mesh, kern, maxiter=500, tol=tol, n_smooth=2, omega=0.6, n_level=n_level, precision=precision,
                    coarse_correction=cc)
    fe = FiniteElement(mesh, kern, sol)
    kern.add_constraints(torch.as_tensor(wl["fixed_dofs"], device="cuda"))
    fe.rhs.copy_(torch.as_tensor(wl["rhs"], device="cuda"))
    return kern, sol, fe


def _modulated(nel, x):
    """The solution with a smooth modulation along x per component: a field the deflation
    space helps with but does not solve."""
    dim = len(nel)
    nn = np.array(nel) + 1
    node = np.arange(int(np.prod(nn)))
    # node index: k + nz (i + nx j) in 3D, i + nx j in 2D
    ix = (node // nn[2]) % nn[0] if dim == 3 else node % nn[0]
    t = np.repeat(np.pi * ix / nel[0], dim)
    y = x.copy()
    for c in range(dim):
        y[c::dim] *= 1.0 + 0.5 * np.cos(t[c::dim] + c)
    return y


CASES = [("cant", (32, 16, 16), 3), ("bridge", (16, 8, 8), 3), ("cant", (24, 16, 8), 3), ("mbb", (64, 32), 3)]


def _wl(kind, nel):
    return (workloads.cantilever3d(*nel) if kind == "cant" else workloads.bridge3d(*nel) if kind == "bridge"
            else workloads.mbb2d(*nel))


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}{c[1]}")
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_deflated_mgcg_matches_oracle(case, precision):
    kind, nel, nl = case
    wl = _wl(kind, nel)
    K0 = unit_K0(len(nel))
    xo, it_plain, _, st = O.mgcg_solve(nel, K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=nl, tol=1e-10)
    assert st == 0
    y = _modulated(nel, xo)
    xd, it_defl, _, st = O.mgcg_solve(nel, K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=nl, tol=1e-10,
                                      deflation=y)
    assert st == 0 and rel(xd, xo) < 1e-8
    cc = _Given(y)
    kern, sol, fe = _problem(wl, nl, precision, cc)
    U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
    assert cc.calls == 1
    assert sol.last_info["status"] == "PF_OK" and res < 1e-10
    slack = 1 if precision == "fp64" else 2
    assert abs(sol.last_info["iterations"] - it_defl) <= slack, (sol.last_info["iterations"], it_defl, it_plain)
    assert rel(U.cpu().numpy(), xo) < 1e-8


def test_exact_field_solves_in_one_iteration():
    """With the solution itself as the field, the deflated start is the solution up to the
    FP32 rounding of Q: a handful of iterations, where the plain solve takes dozens."""
    wl = workloads.cantilever3d(32, 16, 16)
    xo, it_plain, _, _ = O.mgcg_solve((32, 16, 16), unit_K0(3), wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=3,
                                      tol=1e-8)
    kern, sol, fe = _problem(wl, 3, "fp64", _Given(xo), tol=1e-8)
    U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
    assert sol.last_info["status"] == "PF_OK"
    assert sol.last_info["iterations"] <= max(3, it_plain // 4), (sol.last_info["iterations"], it_plain)
    assert rel(U.cpu().numpy(), xo) < 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed_bf16"])
def test_random_field_still_converges(precision):
    """A field with no relation to the solution (white noise) costs at most a few
    iterations, and the solve still meets the tolerance with the plain solution."""
    wl = workloads.cantilever3d(32, 16, 16)
    xo, it_plain, _, _ = O.mgcg_solve((32, 16, 16), unit_K0(3), wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=3,
                                      tol=1e-10)
    y = np.random.default_rng(4).standard_normal(xo.size)
    kern, sol, fe = _problem(wl, 3, precision, _Given(y))
    U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
    assert sol.last_info["status"] == "PF_OK" and res < 1e-10
    assert sol.last_info["iterations"] <= it_plain + 5
    assert rel(U.cpu().numpy(), xo) < 1e-8


def test_deflation_is_set_per_solve_and_cleared():
    """Each solve sets the deflation again after the hierarchy setup (K Q changes with the
    densities); with the correction removed the solver is the plain MGCG again."""
    from pyfantom_b200 import _lib
    wl = workloads.cantilever3d(32, 16, 16)
    xo, it_plain, _, _ = O.mgcg_solve((32, 16, 16), unit_K0(3), wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=3,
                                      tol=1e-10)
    y = _modulated((32, 16, 16), xo)
    cc = _Given(y)
    kern, sol, fe = _problem(wl, 3, "fp64", cc)
    E = torch.as_tensor(wl["E"], device="cuda")
    its = []
    for _ in range(3):
        U, res = sol.solve(fe.rhs, rho=E, use_last=False)
        its.append(sol.last_info["iterations"])
        assert rel(U.cpu().numpy(), xo) < 1e-8
    assert cc.calls == 3 and len(set(its)) == 1
    sol.coarse_correction = None
    U, res = sol.solve(fe.rhs, rho=E, use_last=False)
    assert abs(sol.last_info["iterations"] - it_plain) <= 1
    # explicit clear through the C-ABI
    _lib.check(_lib.load().pf_mg_set_deflation(sol._mg, None, _lib.stream()))
    assert sol.last_info["status"] == "PF_OK"
