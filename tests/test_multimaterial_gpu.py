"""GPU: multi-material SIMP (pyFANTOM/Problem/CUDA/MinimumCompliance.py:326-349, 369-411)
and the multi-constraint OC (Optimizers/CUDA/OC.py:104-127) against the reference.

Fixtures: tests/golden/make_golden.py runs the reference's CPU MinimumCompliance / OC
(same code as the CUDA classes with numpy for cupy) with a direct solver; this library
solves with MGCG to 1e-11, so the trajectory is compared at 1e-6 relative.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel
from pyfantom_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag,kw", [("m2", dict(void=1e-9, penalty=3.0, heavyside=False)),
                                    ("m3", dict(void=1e-9, penalty=3.0, heavyside=False)),
                                    ("m3h", dict(void=1e-6, penalty=2.5, heavyside=True, beta=3.0, eta=0.45))])
def test_penalize_multi_kernel(golden, tag, kw):
    from pyfantom_b200.Problem import simp_params
    g = golden("multimaterial")
    rho = g[tag + "_rho"]
    ne, nm = rho.shape
    E_mul = np.array([1.0, 0.6, 0.3][:nm])
    p = simp_params(kw["penalty"], kw["void"], 1.0, kw.get("beta", 2.0), kw.get("eta", 0.5), kw["heavyside"])
    r = torch.as_tensor(rho.T.copy(), device="cuda")
    E = torch.empty(ne, dtype=torch.float64, device="cuda")
    dE = torch.empty(nm * ne, dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().pf_penalize_multi_f64(ne, nm, _lib.ptr(r), ctypes.byref(p), E_mul.ctypes.data,
                                                 _lib.ptr(E), _lib.ptr(dE), _lib.stream()))
    assert rel(E.cpu().numpy(), g[tag + "_E"]) < 1e-14
    assert rel(dE.cpu().numpy().reshape(nm, ne).T, g[tag + "_dE"]) < 1e-13


def _mbb_two_materials():
    from pyfantom_b200.CUDA import (FiniteElement, MinimumCompliance, MultiGrid, StructuredFilter2D,
                                    StructuredMesh2D, StructuredStiffnessKernel)
    from pyfantom_b200.physics import LinearElasticity
    wl = workloads.mbb2d(48, 16)
    mesh = StructuredMesh2D(48, 16, 48, 16, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    sol = MultiGrid(mesh, kern, maxiter=4000, tol=1e-11, n_smooth=2, omega=0.6, n_level=3)
    fe = FiniteElement(mesh, kern, sol)
    fe.add_dirichlet_boundary_condition(node_ids=torch.as_tensor(wl["left_nodes"], device="cuda"),
                                        dofs=np.array([[1, 0]]), rhs=0.0)
    fe.add_dirichlet_boundary_condition(node_ids=np.array([wl["br_node"]]), dofs=np.array([[0, 1]]), rhs=0.0)
    fe.add_point_forces(forces=np.array([[0.0, -1.0]]), node_ids=np.array([wl["tl_node"]]))
    prob = MinimumCompliance(fe, StructuredFilter2D(mesh, 1.5), E_mul=[1.0, 0.5], void=1e-9, penalty=3.0,
                             volume_fraction=[0.15, 0.15], heavyside=False)
    return prob


def test_two_material_oc_trajectory_matches_reference(golden):
    from pyfantom_b200.CUDA import OC
    g = golden("multimaterial")
    prob = _mbb_two_materials()
    oc = OC(prob, move=0.2)
    assert np.array_equal(prob.get_desvars().cpu().numpy(), g["mbb_x0"])
    assert prob.m() == 2 and prob.N() == 2 * 48 * 16
    assert rel(prob.nabla_f().cpu().numpy(), g["mbb_df0"]) < 1e-8
    f = [float(prob.f())]
    for _ in range(10):
        oc.iter()
        f.append(float(prob.f()))
    f = np.array(f)
    assert abs(f[0] - g["mbb_f"][0]) < 1e-9 * g["mbb_f"][0]
    assert np.abs(f - g["mbb_f"]).max() / g["mbb_f"].min() < 1e-6
    assert np.abs(prob.get_desvars().cpu().numpy() - g["mbb_x10"]).max() < 1e-5
    assert np.abs(prob.g().cpu().numpy() - g["mbb_g10"]).max() < 1e-8
    df10 = prob.nabla_f().cpu().numpy()
    assert np.abs(df10 - g["mbb_df10"]).max() < 1e-5 * np.abs(g["mbb_df10"]).max()
    # thresholded re-solve of the mixture
    out = prob.FEA()
    assert float(out["compliance"]) > 0


def test_single_material_paths_reject_multi():
    from pyfantom_b200.autograd import compliance
    prob = _mbb_two_materials()
    prob.init_desvars()
    with pytest.raises(NotImplementedError):
        compliance(prob.get_desvars(), prob)
