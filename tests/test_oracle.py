"""CPU: the oracle and the host-side restatements against the reference's golden vectors.

The golden fixtures were produced by running the reference pyFANTOM CPU code
(tests/golden/make_golden.py); these tests pin the oracle before it is trusted as the
checker of the CUDA path.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel, unit_K0
from oracle import oracle as O
from pyfantom_b200 import workloads
from pyfantom_b200.geom import _unit_element, cone_weights
from pyfantom_b200.physics import LinearElasticity


@pytest.mark.parametrize("tag", ["h8_nu03", "h8_nu13", "h8_aniso", "q4_nu03", "q4_aniso"])
def test_k0_matches_reference(golden, tag):
    g = golden("k0")
    K = LinearElasticity(E=1.0, nu=float(g[tag + "_nu"])).K(_unit_element(g[tag + "_h"]))
    assert rel(K, g[tag]) < 1e-14


def test_k0_properties():
    for dim in (2, 3):
        K = unit_K0(dim)
        assert np.allclose(K, K.T, atol=1e-15)
        w = np.linalg.eigvalsh(K)
        assert w.min() > -1e-12
        n_rigid = 3 if dim == 2 else 6
        assert np.sum(np.abs(w) < 1e-10) == n_rigid
        # rigid translations are in the null space (row sums per component vanish)
        for d in range(dim):
            t = np.zeros(K.shape[0])
            t[d::dim] = 1.0
            assert np.abs(K @ t).max() < 1e-14


@pytest.mark.parametrize("tag", ["3d", "3d_odd", "2d", "2d_odd"])
def test_operators(golden, tag):
    g = golden("operators")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    K0 = unit_K0(len(nel))
    E, u, cons = g[tag + "_E"], g[tag + "_u"], g[tag + "_cons"]
    assert rel(O.matvec(nel, K0, E, u), g[tag + "_y_free"]) < 1e-13
    assert rel(O.matvec(nel, K0, E, u, cons), g[tag + "_y_con"]) < 1e-13
    assert rel(O.diagonal(nel, K0, E), g[tag + "_diag_free"]) < 1e-13
    assert rel(O.diagonal(nel, K0, E, cons), g[tag + "_diag_con"]) < 1e-13
    assert rel(O.process_dk(nel, K0, u), g[tag + "_dk"]) < 1e-13


def test_mesh_connectivity_matches_reference(golden):
    g = golden("operators")
    import torch
    from pyfantom_b200 import geom
    dev = torch.device("cpu")
    for tag in ["3d", "3d_odd", "2d", "2d_odd"]:
        nel = tuple(int(v) for v in g[tag + "_nel"])
        orig = geom.device
        geom.device = lambda: dev
        try:
            el = geom._structured_elements(np.array(nel)).numpy()
            nodes = geom._structured_nodes(np.array(nel), np.array(nel, dtype=float)).numpy()
        finally:
            geom.device = orig
        assert np.array_equal(el, g[tag + "_elements"])
        assert np.array_equal(nodes, g[tag + "_nodes"])


@pytest.mark.parametrize("tag", ["3d", "2d"])
def test_transfers(golden, tag):
    g = golden("transfers")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    assert np.array_equal(O.restrict(nel, g[tag + "_vf"]), g[tag + "_restricted"])
    assert np.array_equal(O.prolong(nel, g[tag + "_vc"]), g[tag + "_prolonged"])
    # R = P^T
    rng = np.random.default_rng(0)
    vf = rng.standard_normal(O.n_nodes(nel) * len(nel))
    vc = rng.standard_normal(O.n_nodes(O.coarse_nel(nel)) * len(nel))
    assert abs(vc @ O.restrict(nel, vf) - vf @ O.prolong(nel, vc)) < 1e-12 * abs(vc @ O.restrict(nel, vf))


@pytest.mark.parametrize("tag", ["3d", "2d"])
def test_galerkin(golden, tag):
    g = golden("transfers")
    nel = tuple(int(v) for v in g["gal" + tag + "_nel"])
    K0 = unit_K0(len(nel))
    A1 = O.galerkin_l0(nel, K0, g["gal" + tag + "_E"], g["gal" + tag + "_cons"])
    D1 = O.stencil_to_dense(O.coarse_nel(nel), A1)
    assert rel(D1, g["gal" + tag + "_A1"]) < 1e-13
    A2 = O.galerkin_l1p(O.coarse_nel(nel), A1)
    D2 = O.stencil_to_dense(O.coarse_nel(O.coarse_nel(nel)), A2)
    assert rel(D2, g["gal" + tag + "_A2"]) < 1e-13
    assert np.allclose(D1, D1.T, atol=1e-14 * np.abs(D1).max())


@pytest.mark.parametrize("tag", ["3d_r2", "3d_r25", "3d_aniso", "2d_r15", "2d_r3"])
def test_filter(golden, tag):
    g = golden("filters")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    w, off = cone_weights(nel, g[tag + "_h"], float(g[tag + "_r"]))
    assert np.array_equal(off, g[tag + "_offsets"])
    assert rel(w, g[tag + "_weights"]) < 1e-15
    nrm = O.filter_normalizer(nel, w, off)
    assert rel(nrm, g[tag + "_normalizer"]) < 1e-14
    assert rel(O.filter_fwd(nel, w, off, g[tag + "_v"]), g[tag + "_fwd"]) < 1e-14
    assert rel(O.filter_adj(nel, w, off, nrm, g[tag + "_v"]), g[tag + "_adj"]) < 1e-14
    # exact adjoint: <Hx, y> = <x, H^T y>
    rng = np.random.default_rng(3)
    x, y = rng.standard_normal(len(nrm)), rng.standard_normal(len(nrm))
    lhs = O.filter_fwd(nel, w, off, x) @ y
    assert abs(lhs - x @ O.filter_adj(nel, w, off, nrm, y)) < 1e-12 * max(1.0, abs(lhs))


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_oc_bitexact(golden, tag):
    g = golden("oc")
    x = g[tag + "_x"]
    xn, steps = O.oc_update(x, g[tag + "_df"], 1.0 / x.size, float(g[tag + "_vf"]), float(g[tag + "_move"]))
    assert np.array_equal(xn, g[tag + "_xnew"])
    assert 20 <= steps <= 100


@pytest.mark.parametrize("tag", ["plain", "heavy", "emul"])
def test_penalize(golden, tag):
    g = golden("penalize")
    kw = {"plain": dict(penalty=3.0, void=1e-9), "heavy": dict(penalty=3.0, void=1e-9, heavyside=True, beta=4.0, eta=0.4),
          "emul": dict(penalty=2.5, void=1e-6, E_mul=2.0)}[tag]
    assert rel(O.penalize(g["rho"], **kw), g[tag + "_E"]) < 1e-14
    kg = {k: v for k, v in kw.items() if k != "void"}
    assert rel(O.penalize_grad(g["rho"], **kg), g[tag + "_dE"]) < 1e-13


def test_mgcg_oracle_matches_direct_solve(golden):
    g = golden("solve16")
    wl = workloads.cantilever3d(16, 8, 8, 0)
    assert np.array_equal(wl["E"], g["E"]) and np.array_equal(wl["rhs"], g["rhs"])
    K0 = unit_K0(3)
    for nl in (1, 2, 3):
        x, it, res, st = O.mgcg_solve(wl["nel"], K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=nl, tol=1e-10)
        assert st == 0 and res < 1e-10
        r = wl["rhs"] - O.matvec(wl["nel"], K0, wl["E"], x, wl["fixed_dofs"])
        assert np.linalg.norm(r) / np.linalg.norm(wl["rhs"]) < 2e-10
        assert rel(x, g["direct_U"]) < 1e-9
        assert abs(wl["rhs"] @ x - float(g["direct_compliance"])) < 1e-9 * float(g["direct_compliance"])


def test_known_answers_file():
    ka = json.load(open(os.path.join(GOLDEN, "known_answers.json")))
    assert ka["mbb_120x40"]["f_init"] == pytest.approx(1026.8430675962559, rel=1e-15)
    assert ka["mbb_120x40"]["f_iter50"] == pytest.approx(202.13500765477625, rel=1e-15)


def test_workloads():
    wl = workloads.cantilever3d(8, 4, 4, 0)
    assert wl["fixed_dofs"].size == 5 * 5 * 3
    assert np.isclose(wl["rhs"].sum(), -1.0)
    b = workloads.bridge3d(8, 4, 4, 0)
    assert b["fixed_dofs"].size == 2 * 5 * 3
    m = workloads.mbb2d(12, 4)
    assert m["fixed_dofs"].size == 5 + 1


@pytest.mark.parametrize("tag", ["p1", "p2", "p3"])
def test_pgd_projection_matches_reference(golden, tag):
    g = golden("pgd")
    xs = g[tag + "_xs"]
    x, l, steps = O.pgd_project(xs, np.full(xs.size, 1.0 / xs.size), float(g[tag + "_vf"]))
    assert np.array_equal(x, g[tag + "_xnew"]) or rel(x, g[tag + "_xnew"]) < 1e-14
    if tag == "p3":  # clip(xs) already satisfies the constraint: no shift
        assert steps == 0 and l == 0.0
    else:
        assert steps > 20 and l < 0


@pytest.mark.parametrize("tag,m", [("q1", 2), ("q2", 3), ("q3", 2)])
def test_pgd_block_projection_matches_reference(golden, tag, m):
    """m lockstep bisections, one per material block (the reference's m > 1 branch).  The
    shifts are refined to the last bit of the constraint sums, summed here per block and in
    the reference over the whole row, hence 1e-15 rather than equality."""
    g = golden("pgd_multi")
    xs = g[tag + "_xs"].reshape(m, -1)
    ne = xs.shape[1]
    x, l, sweeps = O.pgd_project_multi(xs, np.full((m, ne), 1.0 / ne), g[tag + "_vf"])
    assert np.abs(x.reshape(-1) - g[tag + "_xnew"]).max() < 1e-15
    if tag == "q3":  # clip(xs) satisfies every constraint
        assert sweeps == 0 and np.all(l == 0.0)
    else:  # one block feasible at l = 0: its l2 halves from -1e12 until it underflows
        assert sweeps == 1115 and np.sum(l == 0.0) == 1 and np.all(l <= 0.0)


def test_pgd_golden_trajectory_sane(golden):
    g = golden("pgd")
    f = g["f"]
    assert f[0] == pytest.approx(1026.843067509509, rel=1e-13) and f[-1] < 0.25 * f[0]
    assert g["alpha"].shape == (30,) and np.all(g["alpha"] > 0)
    assert abs(g["x_init"].mean() - 0.5) < 1e-12


@pytest.mark.parametrize("tag,kw", [("m2", dict(void=1e-9, penalty=3.0)), ("m3", dict(void=1e-9, penalty=3.0)),
                                    ("m3h", dict(void=1e-6, penalty=2.5, heavyside=True, beta=3.0, eta=0.45))])
def test_penalize_multi_matches_reference(golden, tag, kw):
    g = golden("multimaterial")
    rho = g[tag + "_rho"]
    E_mul = [1.0, 0.6, 0.3][:rho.shape[1]]
    E, dE = O.penalize_multi(rho, E_mul, **kw)
    assert rel(E, g[tag + "_E"]) < 1e-14
    assert rel(dE, g[tag + "_dE"]) < 1e-13


@pytest.mark.parametrize("tag", ["3d", "2d"])
def test_cg_iterates_match_reference(golden, tag):
    """The oracle's textbook CG takes the reference CG loop's steps: after N iterations from
    x0 = 0 (rtol 0, so neither stops early) the iterates agree."""
    g = golden("cg")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    K0 = unit_K0(len(nel))
    for n in g[tag + "_its"]:
        x, it, _ = O.cg_solve(nel, K0, g[tag + "_E"], g[tag + "_cons"], g[tag + "_rhs"], tol=0.0, maxiter=int(n))
        assert it == int(n)
        assert rel(x, g[f"{tag}_x{int(n)}"]) < 1e-10


def test_cg_stops_at_tolerance_and_solves():
    """Stopping rule of cupyx cg: the first iterate with ||r|| <= tol ||b||."""
    wl = workloads.cantilever3d(8, 4, 4)
    K0 = unit_K0(3)
    x, it, res = O.cg_solve(wl["nel"], K0, wl["E"], wl["fixed_dofs"], wl["rhs"], tol=1e-9, maxiter=5000)
    assert res <= 1e-9
    _, it_prev, res_prev = O.cg_solve(wl["nel"], K0, wl["E"], wl["fixed_dofs"], wl["rhs"], tol=1e-9, maxiter=it - 1)
    assert res_prev > 1e-9
    xm, _, _, _ = O.mgcg_solve(wl["nel"], K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=1, tol=1e-12)
    assert rel(x, xm) < 1e-7


def test_oracle_deflated_pcg():
    """The oracle's deflated PCG (the library's learned coarse-grid correction): with the
    solution as the field it converges in one iteration; with a white-noise field it reaches
    the plain solution to the same tolerance."""
    nel = (16, 8, 8)
    wl = workloads.cantilever3d(*nel)
    K0 = unit_K0(3)
    x, it, _, st = O.mgcg_solve(nel, K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=2, tol=1e-10)
    assert st == 0
    x1, it1, _, st1 = O.mgcg_solve(nel, K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=2, tol=1e-8, deflation=x)
    assert st1 == 0 and it1 == 1 and rel(x1, x) < 1e-8
    y = np.random.default_rng(0).standard_normal(x.size)
    x2, it2, _, st2 = O.mgcg_solve(nel, K0, wl["E"], wl["fixed_dofs"], wl["rhs"], n_level=2, tol=1e-10, deflation=y)
    assert st2 == 0 and abs(it2 - it) <= 3 and rel(x2, x) < 1e-8


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_odd_2d_transfers_and_galerkin(golden, tag):
    """2D grids with odd element counts (coarse grids floor nel / 2): restriction,
    prolongation (where P differs from R^T: a fine node past the last coarse node takes
    that node's value) and the Galerkin levels against the reference's own code."""
    g = golden("odd2d")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    assert np.array_equal(O.restrict(nel, g[tag + "_vf"]), g[tag + "_restricted"])
    assert np.array_equal(O.prolong(nel, g[tag + "_vc"]), g[tag + "_prolonged"])
    K0 = unit_K0(2)
    A1 = O.galerkin_l0(nel, K0, g[tag + "_E"], g[tag + "_cons"])
    D1 = O.stencil_to_dense(O.coarse_nel(nel), A1)
    assert rel(D1, g[tag + "_A1"]) < 1e-13
    A2 = O.galerkin_l1p(O.coarse_nel(nel), A1)
    D2 = O.stencil_to_dense(O.coarse_nel(O.coarse_nel(nel)), A2)
    assert rel(D2, g[tag + "_A2"]) < 1e-13


def test_odd_2d_vcycle_matches_reference(golden):
    """MBB 30x10 with 3 levels (15x5, 7x2, 3x1): one V-cycle from a zero guess on the
    reference's own hierarchy (its _multi_grid) equals the oracle's.  At odd sizes the
    prolongation is not R^T, so the V-cycle is not symmetric and the PCG stagnates: the
    reference's solve stops at maxiter with a relative residual near 1e-3."""
    g = golden("odd2d")
    wl = workloads.mbb2d(30, 10)
    z = O.mg_vcycle((30, 10), unit_K0(2), g["mbb_E"], wl["fixed_dofs"], g["mbb_r"], n_level=3, n_smooth=2,
                    omega=0.45)
    assert rel(z, g["mbb_z"]) < 1e-12
    assert float(g["mbb_res"]) > 1e-4


@pytest.mark.parametrize("tag,w_level", [("w0", (0,)), ("w1", (1,)), ("w01", (0, 1))])
def test_w_cycle_matches_reference(golden, tag, w_level):
    """The lower-case 'w' cycle (a second coarse correction at the levels in w_level) on a
    16x8x8 cantilever with 3 coarse levels: one cycle from a zero guess on the reference's
    own hierarchy, and the MultiGrid solve to 1e-10."""
    g = golden("wcycle")
    nel = (16, 8, 8)
    wl = workloads.cantilever3d(*nel, seed=0)
    assert np.array_equal(wl["rhs"], g["rhs"]) and np.array_equal(wl["E"], g["E"])
    K0 = unit_K0(3)
    z = O.mg_vcycle(nel, K0, g["E"], wl["fixed_dofs"], g[tag + "_r"], n_level=3, n_smooth=2, omega=0.45,
                    w_level=w_level)
    assert rel(z, g[tag + "_z"]) < 1e-12
    zv = O.mg_vcycle(nel, K0, g["E"], wl["fixed_dofs"], g[tag + "_r"], n_level=3, n_smooth=2, omega=0.45)
    assert rel(zv, g[tag + "_z"]) > 1e-3  # the second correction changes the cycle
    x, it, res, st = O.mgcg_solve(nel, K0, g["E"], wl["fixed_dofs"], g["rhs"], n_level=3, tol=1e-10,
                                  w_level=w_level)
    assert st == 0 and res < 1e-10
    assert rel(x, g[tag + "_U"]) < 1e-8


def test_w_cycle_2d_solve_matches_reference(golden):
    g = golden("wcycle")
    wl = workloads.mbb2d(32, 16)
    x, it, res, st = O.mgcg_solve((32, 16), unit_K0(2), g["mbb_E"], wl["fixed_dofs"], wl["rhs"], n_level=3,
                                  tol=1e-10, w_level=(1,))
    assert st == 0 and rel(x, g["mbb_U"]) < 1e-8


def _contrast_field(nel, seed=5):
    """A 0/1 design (smoothed noise thresholded at 40 % volume, E = max(rho^3, 1e-9)) with
    solid slabs at the clamp and at the loaded end: SIMP-like contrast."""
    from scipy.ndimage import gaussian_filter
    g = gaussian_filter(np.random.default_rng(seed).standard_normal(nel), 2.0)
    E = np.maximum((g > np.quantile(g, 0.6)).astype(float) ** 3, 1e-9)
    E[:2] = 1.0
    E[-2:] = 1.0
    return E.reshape(-1).copy()


def test_fixed_jacobi_weight_converges_where_the_schedule_stalls():
    """A fixed Jacobi weight (the library's fixed_omega; no reference counterpart) keeps the
    preconditioner the same in every iteration, as PCG assumes.  On a 0/1 design with 1e-9
    voids the reference's residual-driven schedule stalls (its preconditioner changes while
    the residual falls from 1 to 1e-3), the fixed weight converges; on the smooth cantilever
    it reaches the direct solution in fewer iterations."""
    nel = (32, 16, 16)
    wl = workloads.cantilever3d(*nel)
    E = _contrast_field(nel)
    K0 = unit_K0(3)
    x, it, res, st = O.mgcg_solve(nel, K0, E, wl["fixed_dofs"], wl["rhs"], n_level=3, tol=1e-8, maxiter=600,
                                  fixed_omega=0.5)
    r = wl["rhs"] - O.matvec(nel, K0, E, x, wl["fixed_dofs"])
    assert st == 0 and res < 1e-8 and np.linalg.norm(r) / np.linalg.norm(wl["rhs"]) < 2e-8
    _, it2, res2, st2 = O.mgcg_solve(nel, K0, E, wl["fixed_dofs"], wl["rhs"], n_level=3, tol=1e-8, maxiter=400)
    assert st2 == 1 and res2 > 1e-6
    g = np.load(os.path.join(GOLDEN, "solve16.npz"))
    w16 = workloads.cantilever3d(16, 8, 8, 0)
    xa, ita, _, sta = O.mgcg_solve(w16["nel"], K0, w16["E"], w16["fixed_dofs"], w16["rhs"], n_level=2, tol=1e-10)
    xf, itf, _, stf = O.mgcg_solve(w16["nel"], K0, w16["E"], w16["fixed_dofs"], w16["rhs"], n_level=2, tol=1e-10,
                                   fixed_omega=0.5)
    assert sta == stf == 0 and itf < ita
    assert rel(xf, g["direct_U"]) < 1e-9
