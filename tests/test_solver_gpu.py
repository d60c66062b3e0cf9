"""GPU: V-cycle, MGCG, CG, failure statuses and the SIMP loop against the oracle and the
reference goldens.

Tolerances: the V-cycle is compared with the oracle's V-cycle to 1e-10 relative (same
algorithm, different summation order); solves must reach the requested tolerance with
a true FP64 residual below 2x the tolerance and agree with the oracle / reference direct
solve to 1e-8 relative; compliance 1e-6 relative (the stated parity bar).
"""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, rel, unit_K0
from oracle import oracle as O
from pyfantom_b200 import workloads

pytestmark = pytest.mark.gpu


def setup_problem(wl, n_level, precision="fp64", tol=1e-10, maxiter=500, n_smooth=2, omega=0.6, solver="mg", **mg_kw):
    from pyfantom_b200.CUDA import (CG, FiniteElement, MultiGrid, StructuredMesh2D, StructuredMesh3D,
                                    StructuredStiffnessKernel)
    from pyfantom_b200.physics import LinearElasticity
    nel = wl["nel"]
    phys = LinearElasticity(E=1.0, nu=0.3)
    mesh = StructuredMesh3D(*nel, *nel, physics=phys) if len(nel) == 3 else StructuredMesh2D(*nel, *nel, physics=phys)
    kern = StructuredStiffnessKernel(mesh)
    if solver == "mg":
        sol = MultiGrid(mesh, kern, maxiter=maxiter, tol=tol, n_smooth=n_smooth, omega=omega, n_level=n_level,
                        precision=precision, **mg_kw)
    else:
        sol = CG(kern, maxiter=maxiter, tol=tol)
    fe = FiniteElement(mesh, kern, sol)
    kern.add_constraints(torch.as_tensor(wl["fixed_dofs"], device="cuda"))
    fe.rhs.copy_(torch.as_tensor(wl["rhs"], device="cuda"))
    return mesh, kern, sol, fe


def true_res(kern, U, rhs):
    r = rhs - kern.dot(U)
    return float(torch.linalg.norm(r) / torch.linalg.norm(rhs))


# (16, 8, 40) and (12, 6, 70): two and three z-tiles of the fine matvec (30 owned node
# columns each), the last one partial
@pytest.mark.parametrize("case", [("cant", (16, 8, 8), 2), ("cant", (32, 16, 16), 3), ("bridge", (16, 8, 8), 3),
                                  ("mbb", (64, 32), 3), ("cant", (16, 8, 40), 2), ("bridge", (12, 6, 70), 2)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vcycle_matches_oracle(case, precision):
    kind, nel, nl = case
    wl = (workloads.cantilever3d(*nel) if kind == "cant" else workloads.bridge3d(*nel) if kind == "bridge"
          else workloads.mbb2d(*nel))
    mesh, kern, sol, fe = setup_problem(wl, nl, precision=precision)
    kern.set_rho(torch.as_tensor(wl["E"], device="cuda"))
    sol.setup()
    r = np.random.default_rng(0).standard_normal(kern.shape[0])
    r[wl["fixed_dofs"]] = 0.0
    z = sol.vcycle(torch.as_tensor(r, device="cuda"), omega=0.45).cpu().numpy()
    zr = O.mg_vcycle(nel, unit_K0(len(nel)), wl["E"], wl["fixed_dofs"], r, n_level=nl, n_smooth=2, omega=0.45)
    # the FP32 cycle carries rounding of 1e-7 relative per operation; a wrong node (at a
    # z-tile edge of the fine matvec, say) would be off by O(1)
    assert rel(z, zr) < (1e-10 if precision == "fp64" else 1e-4)


@pytest.mark.parametrize("case", [((16, 8, 8), 2), ((32, 16, 16), 3), ((24, 16, 8), 3), ((16, 8, 40), 2)])
def test_mgcg_matches_oracle(case):
    nel, nl = case
    wl = workloads.cantilever3d(*nel)
    mesh, kern, sol, fe = setup_problem(wl, nl, tol=1e-10)
    U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
    xo, ito, reso, st = O.mgcg_solve(nel, unit_K0(3), wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=nl, tol=1e-10)
    assert sol.last_info["status"] == "PF_OK" and res < 1e-10
    assert abs(sol.last_info["iterations"] - ito) <= 1
    assert true_res(kern, U, fe.rhs) < 2e-10
    assert rel(U.cpu().numpy(), xo) < 1e-8


def test_mgcg_matches_reference_solution(golden):
    g = golden("solve16")
    wl = workloads.cantilever3d(16, 8, 8)
    mesh, kern, sol, fe = setup_problem(wl, 2, tol=1e-10)
    U, res = fe.solve(torch.as_tensor(g["E"], device="cuda"))
    c = float(torch.dot(fe.rhs, U))
    assert abs(c - float(g["direct_compliance"])) < 1e-9 * abs(float(g["direct_compliance"]))
    assert rel(U.cpu().numpy(), g["direct_U"]) < 1e-8
    assert rel(U.cpu().numpy(), g["mg_U"]) < 1e-8


@pytest.mark.parametrize("nel,prec", [((32, 16, 16), "mixed"), ((64, 32), "mixed"), ((32, 16, 16), "mixed_bf16"),
                                      ((64, 32), "mixed_bf16")])
def test_mixed_precision_reaches_fp64_tolerance(nel, prec):
    wl = workloads.cantilever3d(*nel) if len(nel) == 3 else workloads.mbb2d(*nel)
    E = torch.as_tensor(wl["E"], device="cuda")
    _, k64, s64, fe64 = setup_problem(wl, 3, "fp64", tol=1e-8)
    U64, _ = fe64.solve(E)
    _, k32, s32, fe32 = setup_problem(wl, 3, prec, tol=1e-8)
    U32, res = fe32.solve(E)
    assert s32.last_info["status"] == "PF_OK"
    assert true_res(k32, U32, fe32.rhs) < 2e-8
    c64, c32 = float(torch.dot(fe64.rhs, U64)), float(torch.dot(fe32.rhs, U32))
    assert abs(c32 - c64) < 1e-6 * abs(c64)
    assert s32.last_info["iterations"] <= 2 * s64.last_info["iterations"] + 5


def test_warm_start_and_cg():
    wl = workloads.cantilever3d(16, 8, 8)
    E = torch.as_tensor(wl["E"], device="cuda")
    _, kern, sol, fe = setup_problem(wl, 2, tol=1e-9)
    U1, _ = fe.solve(E)
    it1 = sol.last_info["iterations"]
    U2, _ = fe.solve(E)  # warm start from the converged solution
    assert sol.last_info["iterations"] <= 1
    _, kcg, scg, fcg = setup_problem(wl, 2, tol=1e-9, maxiter=5000, solver="cg")
    Ucg, res = fcg.solve(E)
    assert scg.last_info["status"] == "PF_OK" and res < 2e-9
    assert rel(Ucg.cpu().numpy(), U1.cpu().numpy()) < 1e-7
    assert it1 < scg.last_info["iterations"]


@pytest.mark.parametrize("case", [("cant", (8, 4, 4), 1e-9), ("mbb", (32, 16), 1e-8), ("bridge", (12, 6, 4), 1e-10)])
def test_cg_matches_oracle_cg(case):
    """pf_cg_solve (the CG solver) against the oracle's textbook CG, which is pinned to the
    reference CG loop's iterates: same iteration count to within one (rounding of the
    reductions differs), same solution, and the cupyx stopping rule ||r|| <= tol ||b||."""
    kind, nel, tol = case
    wl = (workloads.cantilever3d(*nel) if kind == "cant" else workloads.bridge3d(*nel) if kind == "bridge"
          else workloads.mbb2d(*nel))
    _, kern, sol, fe = setup_problem(wl, 1, tol=tol, maxiter=20000, solver="cg")
    U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
    xo, ito, reso = O.cg_solve(nel, unit_K0(len(nel)), wl["E"], wl["fixed_dofs"], wl["rhs"], tol=tol, maxiter=20000)
    assert sol.last_info["status"] == "PF_OK" and sol.last_info["residual"] <= tol
    assert abs(sol.last_info["iterations"] - ito) <= 1
    assert rel(U.cpu().numpy(), xo) < 1e-6
    assert true_res(kern, U, fe.rhs) < 2 * tol


def test_cg_fixed_iterates_match_reference(golden):
    """With tol = 0 the CG solver runs exactly maxiter iterations: its N-th iterate equals the
    reference CG loop's (golden cg.npz, from x0 = 0)."""
    g = golden("cg")
    for tag, kind in (("3d", "cant"), ("2d", "mbb")):
        nel = tuple(int(v) for v in g[tag + "_nel"])
        wl = workloads.cantilever3d(*nel, seed=3) if kind == "cant" else workloads.mbb2d(*nel)
        for n in g[tag + "_its"]:
            _, kern, sol, fe = setup_problem(wl, 1, tol=0.0, maxiter=int(n), solver="cg")
            fe.rhs.copy_(torch.as_tensor(g[tag + "_rhs"], device="cuda"))
            U, _ = fe.solve(torch.as_tensor(g[tag + "_E"], device="cuda"))
            assert sol.last_info["iterations"] == int(n)
            assert rel(U.cpu().numpy(), g[f"{tag}_x{int(n)}"]) < 1e-9


def test_status_not_converged():
    wl = workloads.cantilever3d(16, 8, 8)
    _, kern, sol, fe = setup_problem(wl, 2, tol=1e-12, maxiter=3)
    U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
    assert sol.last_info["status"] == "PF_NOT_CONVERGED"
    assert sol.last_info["iterations"] == 3 and res > 1e-12


def test_status_nonfinite_input():
    wl = workloads.cantilever3d(16, 8, 8)
    _, kern, sol, fe = setup_problem(wl, 2)
    fe.rhs[5] = float("nan")
    sol.solve(fe.rhs, rho=torch.as_tensor(wl["E"], device="cuda"), use_last=False)
    assert sol.last_info["status"] == "PF_NONFINITE"


def test_status_breakdown_on_zero_operator():
    wl = workloads.cantilever3d(8, 4, 4)
    _, kern, sol, fe = setup_problem(wl, 1, solver="cg")
    kern.reset()  # no constraints, and a zero stiffness: p.Kp = 0
    sol.solve(fe.rhs, rho=torch.zeros(8 * 4 * 4, dtype=torch.float64, device="cuda"), use_last=False)
    assert sol.last_info["status"] == "PF_BREAKDOWN"


def test_bad_level_count_is_rejected():
    """Four halvings of 12x8x8 leave no element on the coarsest level."""
    from pyfantom_b200._lib import PFError
    wl = workloads.cantilever3d(12, 8, 8)
    _, kern, sol, fe = setup_problem(wl, 4)
    with pytest.raises(PFError):
        fe.solve(torch.as_tensor(wl["E"], device="cuda"))


def _mbb_problem(solver="mg"):
    from pyfantom_b200.CUDA import (CG, FiniteElement, MinimumCompliance, MultiGrid, OC, StructuredFilter2D,
                                    StructuredMesh2D, StructuredStiffnessKernel)
    from pyfantom_b200.physics import LinearElasticity
    wl = workloads.mbb2d(120, 40)
    mesh = StructuredMesh2D(120, 40, 120, 40, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    sol = MultiGrid(mesh, kern, maxiter=2000, tol=1e-11, n_smooth=2, omega=0.6, n_level=3)
    fe = FiniteElement(mesh, kern, sol)
    left = torch.as_tensor(wl["left_nodes"], device="cuda")
    fe.add_dirichlet_boundary_condition(node_ids=left, dofs=np.array([[1, 0]]), rhs=0.0)
    fe.add_dirichlet_boundary_condition(node_ids=np.array([wl["br_node"]]), dofs=np.array([[0, 1]]), rhs=0.0)
    fe.add_point_forces(forces=np.array([[0.0, -1.0]]), node_ids=np.array([wl["tl_node"]]))
    filt = StructuredFilter2D(mesh, 1.5)
    prob = MinimumCompliance(fe, filt, E_mul=[1.0], void=1e-9, penalty=3.0, volume_fraction=[0.5], heavyside=False)
    return wl, prob, fe


def test_mbb_setup_matches_reference(golden):
    g = golden("mbb")
    wl, prob, fe = _mbb_problem()
    assert np.array_equal(np.nonzero(fe.kernel.constraints.cpu().numpy())[0], g["cons"])
    assert np.array_equal(fe.rhs.cpu().numpy(), g["rhs"])


def test_mbb_simp_trajectory_matches_reference(golden):
    from pyfantom_b200.CUDA import OC
    g = golden("mbb")
    wl, prob, fe = _mbb_problem()
    oc = OC(prob, move=0.2)
    f = [float(prob.f())]
    for _ in range(50):
        oc.iter()
        f.append(float(prob.f()))
    f = np.array(f)
    assert abs(f[0] - g["f"][0]) < 1e-9 * g["f"][0]
    assert np.abs(f - g["f"]).max() / g["f"].min() < 1e-6
    assert np.abs(prob.get_desvars().cpu().numpy() - g["x50"]).max() < 1e-5
    ka = json.load(open(os.path.join(GOLDEN, "known_answers.json")))["mbb_120x40"]
    assert f[50] == pytest.approx(ka["f_iter50"], rel=1e-6)


def test_sensitivity_matches_reference(golden):
    from pyfantom_b200.CUDA import (FiniteElement, MinimumCompliance, MultiGrid, StructuredFilter3D, StructuredMesh3D,
                                    StructuredStiffnessKernel)
    from pyfantom_b200.physics import LinearElasticity
    g = golden("sensitivity")
    nel = tuple(int(v) for v in g["nel"])
    wl = workloads.bridge3d(*nel, seed=3)
    mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    sol = MultiGrid(mesh, kern, maxiter=1000, tol=1e-12, n_smooth=2, omega=0.6, n_level=1)
    fe = FiniteElement(mesh, kern, sol)
    kern.add_constraints(torch.as_tensor(wl["fixed_dofs"], device="cuda"))
    fe.rhs.copy_(torch.as_tensor(g["rhs"], device="cuda"))
    prob = MinimumCompliance(fe, StructuredFilter3D(mesh, 2.5), E_mul=[1.0], void=1e-9, penalty=3.0,
                             volume_fraction=[0.2], heavyside=False)
    prob.set_desvars(torch.as_tensor(g["x"], device="cuda"))
    assert abs(float(prob.f()) - float(g["f"])) < 1e-9 * abs(float(g["f"]))
    assert rel(prob.nabla_f().cpu().numpy(), g["df"]) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_full_size_cantilever_matches_reference(precision):
    """96x48x48 cantilever (698,691 DOF), 4 levels, tol 1e-8: the reference MultiGrid takes
    83 PCG iterations and reaches compliance 7.472352867980982 (tests/golden/known_answers.json
    records the reference run).  The FP64 drop-in must match the iteration count (+-1); both
    forms must reach a true FP64 residual near 1e-8 and the compliance within 1e-6."""
    wl = workloads.cantilever3d(96, 48, 48)
    _, kern, sol, fe = setup_problem(wl, 4, precision, tol=1e-8, maxiter=1000)
    for _ in range(2):  # repeated solves must agree bitwise (FP64) / stay converged (mixed)
        U, res = fe.solve(torch.as_tensor(wl["E"], device="cuda"))
        sol.last_x0 = None
        info = sol.last_info
        assert info["status"] == "PF_OK"
        if precision == "fp64":
            assert abs(info["iterations"] - 83) <= 1
        else:
            assert info["iterations"] <= 100
        assert true_res(kern, U, fe.rhs) < 1.5e-8
        c = float(torch.dot(fe.rhs, U))
        assert abs(c - 7.472352867980982) < 1e-6 * 7.472352867980982


@pytest.mark.parametrize("prec", ["mixed_bf16", "mixed"])
def test_simp_loop_mixed_forms_track_fp64(prec):
    """The 192x96x96 configuration's loop at 64x32x32: SIMP + OC with the displacement solves
    in the mixed form (FP32 V-cycle, BF16 or FP32 element scales), every iteration's
    stiffness also solved by the FP64 MGCG at the same tolerance: relative compliance error
    below 1e-6 and displacement error below 1e-5 at every iteration."""
    from pyfantom_b200.CUDA import MinimumCompliance, MultiGrid, OC, StructuredFilter3D
    wl = workloads.cantilever3d(64, 32, 32)
    mesh, kern, sol, fe = setup_problem(wl, 4, prec, tol=1e-8, maxiter=1000)
    ref = MultiGrid(mesh, kern, maxiter=1000, tol=1e-8, n_smooth=2, omega=0.6, n_level=4, precision="fp64")
    prob = MinimumCompliance(fe, StructuredFilter3D(mesh, 2.0), E_mul=[1.0], void=1e-9, penalty=3.0,
                             volume_fraction=[0.3], heavyside=False)
    oc = OC(prob, move=0.2)
    for it in range(6):
        if it:
            oc.iter()
        assert sol.last_info["status"] == "PF_OK"
        Ur, _ = ref.solve(fe.rhs, use_last=True)
        cr = float(torch.dot(fe.rhs, Ur))
        assert abs(float(prob.f()) - cr) < 1e-6 * abs(cr)
        assert float(torch.linalg.norm(prob._U - Ur) / torch.linalg.norm(Ur)) < 1e-5


@pytest.mark.parametrize("case", [("mbb", (30, 10), 3), ("mbb", (7, 5), 2), ("mbb", (9, 6), 2),
                                  ("cant", (9, 6, 5), 2), ("cant", (12, 8, 8), 3)])
def test_odd_element_counts_match_oracle(case):
    """Grids whose element counts are odd on some level (every coarse grid floors nel / 2,
    as the reference): level-1 operator, one V-cycle and the first PCG iterates against the
    oracle.  At odd sizes the prolongation is not R^T and the reference's PCG stagnates, so
    iterates are compared, not converged solutions."""
    kind, nel, nl = case
    wl = workloads.cantilever3d(*nel) if kind == "cant" else workloads.mbb2d(*nel)
    K0 = unit_K0(len(nel))
    mesh, kern, sol, fe = setup_problem(wl, nl, tol=1e-14, maxiter=3)
    E = torch.as_tensor(wl["E"], device="cuda")
    kern.set_rho(E)
    sol.setup()
    rng = np.random.default_rng(5)
    cn = tuple(n // 2 for n in nel)
    u = rng.standard_normal(int(np.prod(np.array(cn) + 1)) * len(nel))
    A1 = O.galerkin_l0(nel, K0, wl["E"], wl["fixed_dofs"])
    y = sol.level_matvec(1, torch.as_tensor(u, device="cuda")).cpu().numpy()
    assert rel(y, O.stencil_matvec(cn, A1, u)) < 1e-12
    r = rng.standard_normal(kern.shape[0])
    r[wl["fixed_dofs"]] = 0.0
    z = sol.vcycle(torch.as_tensor(r, device="cuda"), omega=0.45).cpu().numpy()
    zr = O.mg_vcycle(nel, K0, wl["E"], wl["fixed_dofs"], r, n_level=nl, n_smooth=2, omega=0.45)
    assert rel(z, zr) < 1e-10
    U, res = sol.solve(fe.rhs, rho=E, use_last=False)
    xo, ito, _, _ = O.mgcg_solve(nel, K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=nl, tol=1e-14, maxiter=3)
    assert sol.last_info["iterations"] == ito == 3
    assert rel(U.cpu().numpy(), xo) < 1e-9


def test_odd_2d_vcycle_matches_reference_golden(golden):
    """The reference's own V-cycle on the MBB 30x10 hierarchy (15x5, 7x2, 3x1)."""
    g = golden("odd2d")
    wl = workloads.mbb2d(30, 10)
    mesh, kern, sol, fe = setup_problem(wl, 3)
    kern.set_rho(torch.as_tensor(g["mbb_E"], device="cuda"))
    sol.setup()
    z = sol.vcycle(torch.as_tensor(g["mbb_r"], device="cuda"), omega=0.45).cpu().numpy()
    assert rel(z, g["mbb_z"]) < 1e-10


@pytest.mark.parametrize("tag,w_level", [("w0", [0]), ("w1", [1]), ("w01", [0, 1])])
def test_w_cycle_matches_reference_golden(golden, tag, w_level):
    """The reference's lower-case 'w' cycle (second coarse correction at the levels in
    w_level) on a 16x8x8 cantilever with 3 coarse levels: one cycle from a zero guess and
    the MGCG solve to 1e-10 against the reference's own, the iteration count against the
    oracle's."""
    g = golden("wcycle")
    nel = (16, 8, 8)
    wl = workloads.cantilever3d(*nel, seed=0)
    mesh, kern, sol, fe = setup_problem(wl, 3, cycle="w", w_level=w_level)
    E = torch.as_tensor(g["E"], device="cuda")
    kern.set_rho(E)
    sol.setup()
    z = sol.vcycle(torch.as_tensor(g[tag + "_r"], device="cuda"), omega=0.45).cpu().numpy()
    assert rel(z, g[tag + "_z"]) < 1e-10
    U, res = sol.solve(fe.rhs, rho=E, use_last=False)
    x, it, _, _ = O.mgcg_solve(nel, unit_K0(3), g["E"], wl["fixed_dofs"], g["rhs"], n_level=3, tol=1e-10,
                               w_level=w_level)
    assert sol.last_info["status"] == "PF_OK" and abs(sol.last_info["iterations"] - it) <= 1
    assert rel(U.cpu().numpy(), g[tag + "_U"]) < 1e-8
    # the FP32 cycle (element-level level 1) with the same W levels reaches the same solution
    mesh, kern, sol32, fe = setup_problem(wl, 3, precision="mixed", cycle="w", w_level=w_level)
    U32, _ = sol32.solve(fe.rhs, rho=E, use_last=False)
    assert sol32.last_info["status"] == "PF_OK" and rel(U32.cpu().numpy(), g[tag + "_U"]) < 1e-8
    assert abs(sol32.last_info["iterations"] - it) <= 3


def test_w_cycle_2d_matches_reference_golden(golden):
    g = golden("wcycle")
    wl = workloads.mbb2d(32, 16)
    mesh, kern, sol, fe = setup_problem(wl, 3, cycle="w", w_level=1)
    U, res = sol.solve(fe.rhs, rho=torch.as_tensor(g["mbb_E"], device="cuda"), use_last=False)
    assert sol.last_info["status"] == "PF_OK" and rel(U.cpu().numpy(), g["mbb_U"]) < 1e-8


def test_upper_case_w_runs_v_cycles(golden):
    """Only the lower-case 'w' takes the second correction: 'W' (the default) and 'V' give
    the V-cycle."""
    g = golden("wcycle")
    wl = workloads.cantilever3d(16, 8, 8, seed=0)
    r = torch.as_tensor(g["w0_r"], device="cuda")
    zs = []
    for cyc in ("W", "V", "w"):
        mesh, kern, sol, fe = setup_problem(wl, 3, cycle=cyc, w_level=0)
        kern.set_rho(torch.as_tensor(g["E"], device="cuda"))
        sol.setup()
        zs.append(sol.vcycle(r, omega=0.45))
    assert torch.equal(zs[0], zs[1]) and not torch.equal(zs[0], zs[2])



@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("field", ["smooth", "contrast"])
def test_fixed_jacobi_weight_matches_oracle(precision, field):
    """MultiGrid(fixed_omega=0.5): the same weight in every V-cycle (no reference
    counterpart) against the oracle's solve with that weight, on the smooth cantilever and
    on a 0/1 design with 1e-9 voids, where the reference's schedule stalls."""
    from test_oracle import _contrast_field
    nel = (32, 16, 16)
    wl = workloads.cantilever3d(*nel)
    E = wl["E"] if field == "smooth" else _contrast_field(nel)
    mesh, kern, sol, fe = setup_problem(wl, 3, precision=precision, tol=1e-8, maxiter=800, fixed_omega=0.5)
    U, res = sol.solve(fe.rhs, rho=torch.as_tensor(E, device="cuda"), use_last=False)
    xo, ito, _, sto = O.mgcg_solve(nel, unit_K0(3), E, wl["fixed_dofs"], wl["rhs"], n_level=3, tol=1e-8,
                                   maxiter=800, fixed_omega=0.5)
    assert sol.last_info["status"] == "PF_OK" and sto == 0
    # at 1e-9 contrast the iteration count follows the rounding of every sum (the GPU and
    # the oracle add in different orders): 254 against 268 in FP64; the FP32 V-cycle there
    # is a coarser preconditioner and takes about twice the FP64 count (535)
    it = sol.last_info["iterations"]
    if field == "contrast" and precision == "mixed":
        assert it <= 3 * ito, (it, ito)
    else:
        slack = 1 if field == "smooth" and precision == "fp64" else max(3, ito // 10)
        assert abs(it - ito) <= slack, (it, ito)
    assert true_res(kern, U, fe.rhs) < 2e-8
    # the stopping test bounds the residual, not the error: at 1e-9 contrast two solves that
    # both stop at 1e-8 differ by up to cond(K) * 1e-8, and the mixed form's path (twice the
    # iterations, FP32 preconditioner, its own order of every dot product) ends 1e-6..1e-5
    # from the oracle's solution; elsewhere they agree to 1e-6
    bound = 1e-5 if (field == "contrast" and precision == "mixed") else 1e-6
    assert rel(U.cpu().numpy(), xo) < bound


def test_fixed_jacobi_weight_argument_checks():
    from pyfantom_b200 import _lib as L
    wl = workloads.cantilever3d(8, 4, 4)
    for bad in (0.0, -0.5, 2.0):
        with pytest.raises(ValueError):
            setup_problem(wl, 1, fixed_omega=bad)
    mesh, kern, sol, fe = setup_problem(wl, 1)
    cfg = L.pf_mg_config(n_level=1, n_smooth=2, omega=0.6, min_omega=0.4, omega_boost=1.06, coarse_beta=1e-6,
                         precision=0, check_every=4, coarse_op=1, w_mask=0, omega_fixed=-1.0)
    h = ctypes.c_void_p()
    assert L.load().pf_mg_create(kern._op, ctypes.byref(cfg), ctypes.byref(h)) == L.PF_BAD_ARG
