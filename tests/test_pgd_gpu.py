"""GPU: the PGD optimizer (pyFANTOM/Optimizers/CUDA/PGD.py) against the reference.

The projection kernel is compared with the reference's own projections (fixtures written
by tests/golden/make_golden.py from pyFANTOM's CPU PGD, whose code is the CUDA one with
numpy in place of cupy); the statistics pass with numpy; the whole optimizer with the
reference's 30-iteration trajectory on the 120x40 MBB half-beam.  The reference ran with
a direct solver and this library with MGCG to 1e-11, and the step sizes are ratios of
reductions taken in another order, so the trajectory is compared at 1e-6 relative.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel
from oracle import oracle as O
from pyfantom_b200 import _lib

pytestmark = pytest.mark.gpu


def _ws(n):
    return torch.empty(int(_lib.load().pf_pgd_workspace_size(n)), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("tag", ["p1", "p2", "p3"])
def test_projection_matches_reference(golden, tag):
    g = golden("pgd")
    xs = g[tag + "_xs"]
    n = xs.size
    vf = float(g[tag + "_vf"])
    xt = torch.as_tensor(xs, device="cuda")
    dg = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
    out = torch.empty_like(xt)
    h = (ctypes.c_double * 3)()
    w = _ws(n)
    _lib.check(_lib.load().pf_pgd_project_f64(n, _lib.ptr(xt), _lib.ptr(dg), vf, 0.0, 1.0, 1e-8, _lib.ptr(out),
                                              _lib.ptr(w), h, _lib.stream()))
    x_ref, l_ref, steps_ref = O.pgd_project(xs, np.full(n, 1.0 / n), vf)
    assert int(h[1]) == steps_ref and h[0] == l_ref
    assert rel(out.cpu().numpy(), g[tag + "_xnew"]) < 1e-15
    # repeated call: deterministic
    out2 = torch.empty_like(xt)
    _lib.check(_lib.load().pf_pgd_project_f64(n, _lib.ptr(xt), _lib.ptr(dg), vf, 0.0, 1.0, 1e-8, _lib.ptr(out2),
                                              _lib.ptr(w), None, _lib.stream()))
    assert torch.equal(out, out2)


def test_stats_and_step():
    rng = np.random.default_rng(3)
    n = 50001
    x, df, xl, dfl, dl = (rng.standard_normal(n) for _ in range(5))
    t = [torch.as_tensor(a, device="cuda") for a in (x, df, xl, dfl, dl)]
    h = (ctypes.c_double * 8)()
    w = _ws(n)
    _lib.check(_lib.load().pf_pgd_stats_f64(n, _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[2]), _lib.ptr(t[3]),
                                            _lib.ptr(w), h, _lib.stream()))
    s, y = xl - x, dfl - df
    want = [df @ df, np.abs(df).max(), df @ dfl, dfl @ dfl, s @ y, s @ s, y @ y, np.abs(y).max()]
    assert np.allclose(list(h), want, rtol=1e-12, atol=0)
    _lib.check(_lib.load().pf_pgd_stats_f64(n, _lib.ptr(t[0]), _lib.ptr(t[1]), None, None, _lib.ptr(w), h,
                                            _lib.stream()))
    assert np.allclose(list(h)[:2], want[:2], rtol=1e-12) and list(h)[2:] == [0.0] * 6
    d = torch.empty_like(t[0])
    xn = torch.empty_like(t[0])
    _lib.check(_lib.load().pf_pgd_step_f64(n, _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[4]), 0.7, 0.3, _lib.ptr(d),
                                           _lib.ptr(xn), _lib.stream()))
    assert rel(d.cpu().numpy(), -df + 0.7 * dl) < 1e-15
    assert rel(xn.cpu().numpy(), x + 0.3 * (-df + 0.7 * dl)) < 1e-15
    assert _lib.load().pf_pgd_stats_f64(n, _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[2]), None, _lib.ptr(w), h,
                                        _lib.stream()) == _lib.PF_BAD_ARG


def test_pgd_trajectory_matches_reference(golden):
    from test_solver_gpu import _mbb_problem
    from pyfantom_b200.CUDA import PGD
    g = golden("pgd")
    wl, prob, fe = _mbb_problem()
    pgd = PGD(prob)  # initialises the design (uniform volume fraction) and projects it
    # the uniform design sits on the constraint: the reference's sum came out a rounding
    # error above the volume fraction (a shift of 2e-15), this one exactly on it
    assert rel(prob.get_desvars().cpu().numpy(), g["x_init"]) < 1e-12
    f, alpha, change = [], [], []
    for it in range(30):
        pgd.iter()
        f.append(float(pgd.last_f))
        alpha.append(pgd.last_alpha)
        change.append(pgd.change)
        if it in (0, 1):
            assert np.abs(prob.get_desvars().cpu().numpy() - g[f"x{it + 1}"]).max() < 1e-9
    f, alpha = np.array(f), np.array(alpha)
    assert abs(f[0] - g["f"][0]) < 1e-9 * g["f"][0]
    assert np.abs(f - g["f"]).max() / g["f"].min() < 1e-6
    # the solves differ at their 1e-11 tolerance (MGCG here, a direct solve in the reference),
    # and the Barzilai-Borwein step s.s / s.y divides differences of nearly equal vectors, so
    # step sizes agree to 2e-11 at the first iteration, 3e-8 at the tenth, 6e-6 at worst
    ra = np.abs(alpha - g["alpha"]) / np.abs(g["alpha"])
    assert ra[0] < 1e-9 and ra[:10].max() < 1e-6 and ra.max() < 1e-4, ra
    assert np.abs(prob.get_desvars().cpu().numpy() - g["x30"]).max() < 1e-5
    assert pgd.logs()["objective"] == pytest.approx(g["f"][-1], rel=1e-6)
    assert not pgd.converged() or pgd.change <= pgd.change_tol


@pytest.mark.parametrize("tag,m", [("q1", 2), ("q2", 3), ("q3", 2)])
def test_block_projection_matches_reference(golden, tag, m):
    """One volume constraint per material block: the reference's lockstep bisection
    (fixtures from its project_to_feasible with m > 1).  q1 and q2 hold a block that is
    feasible at l = 0, which keeps the loop going until its l2 underflows (1115 sweeps);
    q3 is feasible everywhere (clip(xs)).  The final shifts are refined to the last bit of
    the constraint sums, whose order differs from the reference's, hence 1e-14 on x."""
    g = golden("pgd_multi")
    xs = g[tag + "_xs"]
    ne = xs.size // m
    vf = np.ascontiguousarray(g[tag + "_vf"], dtype=np.float64)
    dgb = np.full((m, ne), 1.0 / ne)
    xt = torch.as_tensor(xs, device="cuda")
    dg = torch.as_tensor(dgb, device="cuda")
    out = torch.empty_like(xt)
    lib = _lib.load()
    w = torch.empty(int(lib.pf_pgd_multi_workspace_size(ne, m)), dtype=torch.float64, device="cuda")
    h = (ctypes.c_double * (2 + m))()
    _lib.check(lib.pf_pgd_project_multi_f64(ne, m, _lib.ptr(xt), _lib.ptr(dg), vf.ctypes.data, 0.0, 1.0, 1e-8,
                                            _lib.ptr(out), _lib.ptr(w), h, _lib.stream()))
    x_ref, l_ref, sweeps_ref = O.pgd_project_multi(xs.reshape(m, ne), dgb, vf)
    assert int(h[0]) == sweeps_ref and bool(h[1]) == (sweeps_ref == 0)
    assert np.allclose(list(h)[2:], l_ref, rtol=1e-13, atol=0)
    assert np.abs(out.cpu().numpy() - g[tag + "_xnew"]).max() < 1e-14
    assert np.abs(out.cpu().numpy() - x_ref.reshape(-1)).max() < 1e-14
    # no host buffer: refused (the sweep count is only known on the host)
    assert lib.pf_pgd_project_multi_f64(ne, m, _lib.ptr(xt), _lib.ptr(dg), vf.ctypes.data, 0.0, 1.0, 1e-8,
                                        _lib.ptr(out), _lib.ptr(w), None, _lib.stream()) == _lib.PF_BAD_ARG


def test_block_projection_with_one_block_is_the_single_projection(golden):
    g = golden("pgd")
    xs = g["p2_xs"]
    n = xs.size
    vf = np.array([float(g["p2_vf"])])
    xt = torch.as_tensor(xs, device="cuda")
    dg = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
    lib = _lib.load()
    a, b = torch.empty_like(xt), torch.empty_like(xt)
    h1, h2 = (ctypes.c_double * 3)(), (ctypes.c_double * 3)()
    _lib.check(lib.pf_pgd_project_f64(n, _lib.ptr(xt), _lib.ptr(dg), float(vf[0]), 0.0, 1.0, 1e-8, _lib.ptr(a),
                                      _lib.ptr(_ws(n)), h1, _lib.stream()))
    w = torch.empty(int(lib.pf_pgd_multi_workspace_size(n, 1)), dtype=torch.float64, device="cuda")
    _lib.check(lib.pf_pgd_project_multi_f64(n, 1, _lib.ptr(xt), _lib.ptr(dg), vf.ctypes.data, 0.0, 1.0, 1e-8,
                                            _lib.ptr(b), _lib.ptr(w), h2, _lib.stream()))
    assert torch.equal(a, b) and h1[0] == h2[2] and h1[1] == h2[0]


def test_two_material_pgd_trajectory_matches_reference(golden):
    """PGD on the 2-material MBB half-beam (48x16, volume fractions 0.15 / 0.15) for 10
    iterations against the reference's (direct solve there, MGCG to 1e-11 here)."""
    from test_multimaterial_gpu import _mbb_two_materials
    from pyfantom_b200.CUDA import PGD
    g = golden("pgd_multi")
    prob = _mbb_two_materials()
    pgd = PGD(prob)
    assert np.abs(prob.get_desvars().cpu().numpy() - g["mbb_x_init"]).max() < 1e-12
    f, alpha = [], []
    for it in range(10):
        pgd.iter()
        f.append(float(pgd.last_f))
        alpha.append(pgd.last_alpha)
        if it in (0, 1):
            assert np.abs(prob.get_desvars().cpu().numpy() - g[f"mbb_x{it + 1}"]).max() < 1e-9
    f, alpha = np.array(f), np.array(alpha)
    assert abs(f[0] - g["mbb_f"][0]) < 1e-9 * g["mbb_f"][0]
    assert np.abs(f - g["mbb_f"]).max() / g["mbb_f"].min() < 1e-6
    ra = np.abs(alpha - g["mbb_alpha"]) / np.abs(g["mbb_alpha"])
    assert ra[0] < 1e-9 and ra.max() < 1e-4, ra
    assert np.abs(prob.get_desvars().cpu().numpy() - g["mbb_x10"]).max() < 1e-5
    assert np.abs(prob.g().cpu().numpy() - g["mbb_g10"]).max() < 1e-8
    assert len(pgd.last_projection["l"]) == 2
