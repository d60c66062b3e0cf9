"""GPU: the differentiable compliance (hand-written adjoint kernel) against the reference's
sensitivity and against central finite differences.

Finite differences use step 1e-6 in FP64 on 32 randomly chosen elements of the 128x64x64
bridge.  Each perturbed compliance is evaluated as f.U + r.U (r = f - K U), which removes
the first-order effect of the solve tolerance; what remains is FP64 rounding in the dot
products (about 1e-15 of c against a difference of about 1e-11 of c), so the test bar is
1e-3 relative per element plus 1e-5 of the largest sensitivity.
"""
import numpy as np
import pytest
import torch

from conftest import rel
from pyfantom_b200 import workloads

pytestmark = pytest.mark.gpu


def _bridge_problem(nel, seed, n_level, tol):
    from pyfantom_b200.CUDA import (FiniteElement, MinimumCompliance, MultiGrid, StructuredFilter3D,
                                    StructuredMesh3D, StructuredStiffnessKernel)
    from pyfantom_b200.physics import LinearElasticity
    wl = workloads.bridge3d(*nel, seed=seed)
    mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    sol = MultiGrid(mesh, kern, maxiter=2000, tol=tol, n_smooth=2, omega=0.6, n_level=n_level)
    fe = FiniteElement(mesh, kern, sol)
    fe.add_dirichlet_boundary_condition(node_ids=torch.as_tensor(wl["fixed_nodes"], device="cuda"), rhs=0.0)
    fe.add_point_forces(forces=wl["load_forces"], node_ids=torch.as_tensor(wl["load_nodes"], device="cuda"))
    prob = MinimumCompliance(fe, StructuredFilter3D(mesh, 2.5), E_mul=[1.0], void=1e-9, penalty=3.0,
                             volume_fraction=[0.2], heavyside=False)
    return wl, prob, fe, kern


def test_adjoint_matches_reference_sensitivity(golden):
    from pyfantom_b200.autograd import compliance, volume
    g = golden("sensitivity")
    nel = tuple(int(v) for v in g["nel"])
    wl, prob, fe, kern = _bridge_problem(nel, 3, 1, 1e-12)
    assert np.array_equal(fe.rhs.cpu().numpy(), g["rhs"])
    x = torch.as_tensor(g["x"], device="cuda").requires_grad_(True)
    c = compliance(x, prob)
    c.backward()
    assert abs(float(c) - float(g["f"])) < 1e-9 * abs(float(g["f"]))
    assert rel(x.grad.cpu().numpy(), g["df"]) < 1e-8
    # same result as the problem's own sensitivity pipeline
    prob.set_desvars(x.detach())
    assert rel(x.grad.cpu().numpy(), prob.nabla_f().cpu().numpy()) < 1e-12
    x.grad = None
    v = volume(x, prob)
    v.backward()
    assert abs(float(v) - float(g["x"].mean())) < 1e-12
    assert torch.allclose(x.grad, prob.nabla_g())


def test_adjoint_heaviside_matches_problem_gradient():
    from pyfantom_b200.autograd import compliance
    wl, prob, fe, kern = _bridge_problem((16, 8, 8), 1, 2, 1e-12)
    prob.heavyside, prob.beta, prob.eta = True, 3.0, 0.45
    x = torch.as_tensor(wl["x"], device="cuda").requires_grad_(True)
    compliance(x, prob).backward()
    prob.set_desvars(x.detach())
    assert rel(x.grad.cpu().numpy(), prob.nabla_f().cpu().numpy()) < 1e-12


def test_adjoint_central_differences_bridge_128x64x64():
    from pyfantom_b200.autograd import compliance
    wl, prob, fe, kern = _bridge_problem((128, 64, 64), 0, 5, 1e-10)
    x0 = torch.as_tensor(wl["x"], device="cuda")
    x = x0.clone().requires_grad_(True)
    compliance(x, prob).backward()
    grad = x.grad.cpu().numpy()

    def energy_compliance(xv):
        E = prob.penalize(prob.filter.dot(xv))
        U, _ = fe.solve(E)  # warm-started from the previous solution
        kern.set_rho(E)
        r = fe.rhs - kern.dot(U)
        return float(torch.dot(fe.rhs, U) + torch.dot(r, U))

    rng = np.random.default_rng(2024)
    idx = rng.choice(x0.numel(), size=32, replace=False)
    h = 1e-6
    gmax = np.abs(grad).max()
    for i in idx:
        xp, xm = x0.clone(), x0.clone()
        xp[i] += h
        xm[i] -= h
        fd = (energy_compliance(xp) - energy_compliance(xm)) / (2 * h)
        assert abs(fd - grad[i]) < 1e-3 * abs(grad[i]) + 1e-5 * gmax, (i, fd, grad[i])
