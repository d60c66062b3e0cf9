"""GPU: the direct solver SPSOLVE (pyFANTOM/solvers/CUDA/_solvers.py:245-328) against the
reference's own direct solves (fixtures from tests/golden/make_golden.py) and the
reference's config-1 MBB trajectory, which ran with SPSOLVE."""
import json
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, rel
from pyfantom_b200 import workloads

pytestmark = pytest.mark.gpu


def test_direct_matches_reference_direct_solve(golden):
    from pyfantom_b200.CUDA import (FiniteElement, SPSOLVE, StructuredMesh3D, StructuredStiffnessKernel)
    from pyfantom_b200.physics import LinearElasticity
    g = golden("solve16")
    wl = workloads.cantilever3d(16, 8, 8)
    mesh = StructuredMesh3D(16, 8, 8, 16, 8, 8, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    fe = FiniteElement(mesh, kern, SPSOLVE(kern))
    fe.add_dirichlet_boundary_condition(node_ids=torch.as_tensor(wl["fixed_nodes"], device="cuda"), rhs=0.0)
    fe.add_point_forces(forces=wl["load_forces"], node_ids=torch.as_tensor(wl["load_nodes"], device="cuda"))
    U, res = fe.solve(torch.as_tensor(g["E"], device="cuda"))
    assert res < 1e-12
    assert rel(U.cpu().numpy(), g["direct_U"]) < 1e-11
    c = float(torch.dot(fe.rhs, U))
    assert abs(c - float(g["direct_compliance"])) < 1e-12 * abs(float(g["direct_compliance"]))
    # repeated solve: same result, constrained entries keep the right-hand side
    U2, _ = fe.solver.solve(fe.rhs)
    assert torch.equal(U, U2)
    con = kern.constraints
    assert torch.equal(U[con], fe.rhs[con])


def test_direct_mbb_trajectory_matches_reference(golden):
    from test_solver_gpu import _mbb_problem
    from pyfantom_b200.CUDA import OC, SPSOLVE
    g = golden("mbb")
    wl, prob, fe = _mbb_problem()
    fe.solver = SPSOLVE(fe.kernel)
    oc = OC(prob, move=0.2)
    f = [float(prob.f())]
    for _ in range(50):
        oc.iter()
        f.append(float(prob.f()))
    f = np.array(f)
    # both sides are direct solves (dense Cholesky here, sparse LU in the reference): they
    # agree to the rounding of a condition number near 1e6 (1.3e-11 relative at iteration 0)
    assert abs(f[0] - g["f"][0]) < 1e-10 * g["f"][0]
    assert np.abs(f - g["f"]).max() / g["f"].min() < 1e-7
    assert np.abs(prob.get_desvars().cpu().numpy() - g["x50"]).max() < 1e-6
    ka = json.load(open(os.path.join(GOLDEN, "known_answers.json")))["mbb_120x40"]
    assert f[50] == pytest.approx(ka["f_iter50"], rel=1e-7)


def test_direct_rejects_oversize():
    from pyfantom_b200._lib import PFError
    from pyfantom_b200.CUDA import SPSOLVE, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    mesh = StructuredMesh3D(20, 20, 20, 20, 20, 20, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    sol = SPSOLVE(kern)
    rhs = torch.ones(kern.shape[0], dtype=torch.float64, device="cuda")
    with pytest.raises(PFError, match="exceed"):
        sol.solve(rhs, rho=torch.ones(8000, dtype=torch.float64, device="cuda"))
