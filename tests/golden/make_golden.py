"""Generate golden fixtures by running the reference pyFANTOM CPU path in this container.

Usage:  PYFANTOM_REFERENCE=<reference checkout> python tests/golden/make_golden.py [--big]

Writes ``tests/golden/*.npz`` (small arrays) and ``tests/golden/known_answers.json``.
Every array is produced by the reference's own code (numba kernels and Python classes
under pyFANTOM/{physics,geom/CPU,stiffness/CPU,core/CPU,solvers/CPU,Problem/CPU,
Optimizers/CPU}); inputs are seeded.  ``--big`` also runs the reference MultiGrid solve
on the 96x48x48 cantilever (about a minute on 8 cores) and records its compliance.

The reference tree is only read here; the committed fixtures are what the tests use.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
warnings.filterwarnings("ignore")

import _refshim  # noqa: E402

_refshim.install()

from pyFANTOM.physics.LinearElasticity import LinearElasticity  # noqa: E402
from pyFANTOM.geom.CPU._mesh import StructuredMesh2D, StructuredMesh3D  # noqa: E402
from pyFANTOM.geom.CPU._filters import StructuredFilter2D, StructuredFilter3D  # noqa: E402
from pyFANTOM.stiffness.CPU import StructuredStiffnessKernel  # noqa: E402
from pyFANTOM.core.CPU._mgm import (apply_restriction, apply_prolongation,  # noqa: E402
                                    get_restricted_l0, get_restricted_l1p)
from pyFANTOM.solvers.CPU._solvers import MultiGrid, SPSOLVE, cg as ref_cg  # noqa: E402
from pyFANTOM.FiniteElement.CPU.FiniteElement import FiniteElement  # noqa: E402
from pyFANTOM.Problem.CPU.MinimumCompliance import MinimumCompliance  # noqa: E402
from pyFANTOM.Optimizers.CPU.OC import OC  # noqa: E402
from pyfantom_b200 import workloads  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}.npz ({os.path.getsize(path)/1024:.1f} KB)")


def k0_goldens():
    out = {}
    for tag, (n, h, nu) in {
        "h8_nu03": ((1, 1, 1), (1.0, 1.0, 1.0), 0.3),
        "h8_nu13": ((1, 1, 1), (1.0, 1.0, 1.0), 1.0 / 3.0),
        "h8_aniso": ((1, 1, 1), (1.0, 0.5, 2.0), 0.3),
    }.items():
        m = StructuredMesh3D(*n, *h, physics=LinearElasticity(E=1.0, nu=nu))
        out[tag] = np.asarray(m.K_single)
        out[tag + "_h"] = np.array(h)
        out[tag + "_nu"] = np.array(nu)
    for tag, (h, nu) in {"q4_nu03": ((1.0, 1.0), 0.3), "q4_aniso": ((1.0, 0.5), 1.0 / 3.0)}.items():
        m = StructuredMesh2D(1, 1, *h, physics=LinearElasticity(E=1.0, nu=nu))
        out[tag] = np.asarray(m.K_single)
        out[tag + "_h"] = np.array(h)
        out[tag + "_nu"] = np.array(nu)
    save("k0", **out)


def operator_goldens():
    """matvec (with and without Dirichlet rows), diagonal and -u_e^T K0 u_e."""
    rng = np.random.default_rng(1234)
    out = {}
    cases = {"3d": ((6, 4, 8), 3), "3d_odd": ((5, 3, 7), 3), "2d": ((6, 4), 2), "2d_odd": ((7, 5), 2)}
    for tag, (nel, dof) in cases.items():
        if dof == 3:
            mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        else:
            mesh = StructuredMesh2D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        n_nodes = mesh.nodes.shape[0]
        nel_total = mesh.elements.shape[0]
        E = rng.uniform(1e-3, 1.0, nel_total)
        u = rng.standard_normal(n_nodes * dof)
        kern = StructuredStiffnessKernel(mesh)
        kern.set_rho(E)
        y_free = np.array(kern.dot(u))
        d_free = np.array(kern.diagonal())
        dk = np.array(kern.process_grad(u))
        # Dirichlet set: every DOF on the x == 0 face plus a random sprinkle of single DOFs
        x0 = np.where(mesh.nodes[:, 0] == 0)[0]
        cons = np.concatenate([(x0[:, None] * dof + np.arange(dof)).reshape(-1),
                               rng.choice(n_nodes * dof, size=max(3, n_nodes // 10), replace=False)])
        cons = np.unique(cons)
        kern.add_constraints(cons)
        y_con = np.array(kern.dot(u))
        d_con = np.array(kern.diagonal())
        out.update({f"{tag}_nel": np.array(nel), f"{tag}_E": E, f"{tag}_u": u, f"{tag}_y_free": y_free,
                    f"{tag}_diag_free": d_free, f"{tag}_dk": dk, f"{tag}_cons": cons,
                    f"{tag}_y_con": y_con, f"{tag}_diag_con": d_con,
                    f"{tag}_elements": np.asarray(mesh.elements), f"{tag}_nodes": np.asarray(mesh.nodes)})
    save("operators", **out)


def transfer_goldens():
    """Restriction / prolongation and the Galerkin coarse operators (as dense matrices)."""
    rng = np.random.default_rng(99)
    out = {}
    for tag, nel, dof in [("3d", (8, 4, 6), 3), ("2d", (8, 6), 2)]:
        nel_a = np.array(nel, dtype=np.int32)
        nf = int(np.prod(nel_a + 1))
        nc = int(np.prod(nel_a // 2 + 1))
        vf = rng.standard_normal(nf * dof)
        vc = rng.standard_normal(nc * dof)
        out[f"{tag}_nel"] = nel_a
        out[f"{tag}_vf"] = vf
        out[f"{tag}_vc"] = vc
        out[f"{tag}_restricted"] = np.array(apply_restriction(vf, nel_a, dof))
        out[f"{tag}_prolonged"] = np.array(apply_prolongation(vc, nel_a, dof))
    # Galerkin hierarchy with Dirichlet rows: level 1 from the fine operator, level 2 from level 1
    for tag, nel, dof in [("3d", (8, 4, 4), 3), ("2d", (8, 8), 2)]:
        if dof == 3:
            mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        else:
            mesh = StructuredMesh2D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        kern = StructuredStiffnessKernel(mesh)
        E = rng.uniform(1e-3, 1.0, mesh.elements.shape[0])
        kern.set_rho(E)
        x0 = np.where(mesh.nodes[:, 0] == 0)[0]
        cons = np.unique(np.concatenate([(x0[:, None] * dof + np.arange(dof)).reshape(-1),
                                         rng.choice(mesh.nodes.shape[0] * dof, size=5, replace=False)]))
        kern.add_constraints(cons)
        A1 = get_restricted_l0(mesh, kern)
        A2 = get_restricted_l1p(A1, mesh.nel // 2, dof)
        out[f"gal{tag}_nel"] = np.array(nel)
        out[f"gal{tag}_E"] = E
        out[f"gal{tag}_cons"] = cons
        out[f"gal{tag}_A1"] = A1.toarray()
        out[f"gal{tag}_A2"] = A2.toarray()
    save("transfers", **out)


def filter_goldens():
    rng = np.random.default_rng(7)
    out = {}
    for tag, nel, h, r in [("3d_r2", (7, 5, 6), (1, 1, 1), 2.0), ("3d_r25", (9, 6, 5), (1, 1, 1), 2.5),
                           ("3d_aniso", (6, 6, 4), (1.0, 0.5, 1.0), 1.5),
                           ("2d_r15", (12, 8), (1, 1), 1.5), ("2d_r3", (10, 9), (1, 1), 3.0)]:
        if len(nel) == 3:
            lx = tuple(n * hh for n, hh in zip(nel, h))
            mesh = StructuredMesh3D(*nel, *lx, physics=LinearElasticity())
            filt = StructuredFilter3D(mesh, r)
        else:
            lx = tuple(n * hh for n, hh in zip(nel, h))
            mesh = StructuredMesh2D(*nel, *lx, physics=LinearElasticity())
            filt = StructuredFilter2D(mesh, r)
        v = rng.uniform(0, 1, int(np.prod(nel)))
        out[f"{tag}_nel"] = np.array(nel)
        out[f"{tag}_h"] = np.array(h, dtype=np.float64)
        out[f"{tag}_r"] = np.array(r)
        out[f"{tag}_v"] = v
        out[f"{tag}_fwd"] = np.array(filt.dot(v))
        out[f"{tag}_adj"] = np.array(filt._rmatvec(v))
        out[f"{tag}_normalizer"] = np.array(filt.normalizer)
        out[f"{tag}_weights"] = np.array(filt.weights)
        out[f"{tag}_offsets"] = np.array(filt.offsets)
    save("filters", **out)


class _FixedProblem:
    """Minimal Problem stand-in that exposes fixed (x, df, dg) to the reference OC."""

    def __init__(self, x, df, vf):
        self.x = x.copy()
        self.df = df
        self.vf = vf
        self.dg = np.full_like(x, 1.0 / x.size)
        self.new = None

    def init_desvars(self):
        return None

    def is_independent(self):
        return True

    def get_desvars(self):
        return self.x

    def f(self, rho=None):
        return 1.0

    def m(self):
        return 1

    def constraint_map(self):
        return 1

    def bounds(self):
        return (0, 1.0)

    def nabla_g(self):
        return self.dg

    def nabla_f(self):
        return self.df

    def g(self, rho=None):
        r = self.x if rho is None else rho
        return (self.dg.reshape(1, -1) @ r.reshape(-1, 1)).reshape(-1) - self.vf

    def set_desvars(self, x):
        self.new = x.copy()


def oc_goldens():
    rng = np.random.default_rng(5)
    out = {}
    for tag, n, vf, move in [("a", 4800, 0.5, 0.2), ("b", 6000, 0.3, 0.2), ("c", 3000, 0.2, 0.05)]:
        x = np.clip(rng.uniform(0.0, 1.0, n), 0, 1)
        df = -np.abs(rng.standard_normal(n)) * rng.uniform(0.01, 10.0)
        if tag == "c":
            df[::7] = 0.0
        prob = _FixedProblem(x, df, vf)
        oc = OC(prob, move=move)
        oc.iter()
        out[f"{tag}_x"] = x
        out[f"{tag}_df"] = df
        out[f"{tag}_vf"] = np.array(vf)
        out[f"{tag}_move"] = np.array(move)
        out[f"{tag}_xnew"] = prob.new
    save("oc", **out)


def penalize_goldens():
    """penalize / penalize_grad (single material) with and without Heaviside projection."""
    mesh = StructuredMesh2D(4, 2, 4, 2, physics=LinearElasticity())
    kern = StructuredStiffnessKernel(mesh)
    fe = FiniteElement(mesh, kern, SPSOLVE(kern))
    filt = StructuredFilter2D(mesh, 1.5)
    rng = np.random.default_rng(11)
    rho = rng.uniform(0.0, 1.0, 1000)
    out = {"rho": rho}
    for tag, kw in {"plain": dict(void=1e-9, penalty=3.0, heavyside=False),
                    "heavy": dict(void=1e-9, penalty=3.0, heavyside=True, beta=4.0, eta=0.4),
                    "emul": dict(void=1e-6, penalty=2.5, heavyside=False, E_mul=[2.0])}.items():
        prob = MinimumCompliance(fe, filt, volume_fraction=[0.5], **kw)
        out[f"{tag}_E"] = np.array(prob.penalize(rho))
        out[f"{tag}_dE"] = np.array(prob.penalize_grad(rho))
    save("penalize", **out)


def multimaterial_goldens():
    """Multi-material SIMP: penalize / penalize_grad for 2 and 3 materials (plain and
    Heaviside), and 10 OC iterations of a 2-material MBB half-beam (48x16, direct solve)."""
    mesh = StructuredMesh2D(4, 2, 4, 2, physics=LinearElasticity())
    kern = StructuredStiffnessKernel(mesh)
    fe = FiniteElement(mesh, kern, SPSOLVE(kern))
    filt = StructuredFilter2D(mesh, 1.5)
    rng = np.random.default_rng(17)
    out = {}
    for tag, nm, kw in [("m2", 2, dict(void=1e-9, penalty=3.0, heavyside=False)),
                        ("m3", 3, dict(void=1e-9, penalty=3.0, heavyside=False)),
                        ("m3h", 3, dict(void=1e-6, penalty=2.5, heavyside=True, beta=3.0, eta=0.45))]:
        E_mul = [1.0, 0.6, 0.3][:nm]
        prob = MinimumCompliance(fe, filt, E_mul=E_mul, volume_fraction=[0.2] * nm, **kw)
        rho = rng.uniform(0.0, 1.0, (500, nm))
        out[f"{tag}_rho"] = rho
        out[f"{tag}_E"] = np.array(prob.penalize(rho))
        out[f"{tag}_dE"] = np.array(prob.penalize_grad(rho))
    wl = workloads.mbb2d(48, 16)
    _, kern2, fe2, _ = _simp_setup(wl, lambda m, k: SPSOLVE(k), 1.5, 0.3)
    filt2 = StructuredFilter2D(fe2.mesh, 1.5)
    prob = MinimumCompliance(fe2, filt2, E_mul=[1.0, 0.5], void=1e-9, penalty=3.0, volume_fraction=[0.15, 0.15],
                             heavyside=False)
    oc = OC(prob, move=0.2)
    out["mbb_x0"] = np.array(prob.get_desvars())
    out["mbb_df0"] = np.array(prob.nabla_f())
    f = [float(prob.f())]
    for _ in range(10):
        oc.iter()
        f.append(float(prob.f()))
    out["mbb_f"] = np.array(f)
    out["mbb_x10"] = np.array(prob.get_desvars())
    out["mbb_df10"] = np.array(prob.nabla_f())
    out["mbb_g10"] = np.array(prob.g())
    print(f"multi-material mbb: f0={f[0]!r} f10={f[-1]!r}")
    save("multimaterial", **out)


def _simp_setup(wl, solver_factory, r_min, vf, void=1e-9, penalty=3.0):
    nel = wl["nel"]
    if wl["dim"] == 3:
        mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        filt = StructuredFilter3D(mesh, r_min)
    else:
        mesh = StructuredMesh2D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        filt = StructuredFilter2D(mesh, r_min)
    kern = StructuredStiffnessKernel(mesh)
    solver = solver_factory(mesh, kern)
    fe = FiniteElement(mesh, kern, solver)
    dof = wl["dof"]
    fixed = wl["fixed_dofs"]
    nodes = np.unique(fixed // dof)
    mask = np.zeros((nodes.size, dof), dtype=np.int64)
    for d in range(dof):
        mask[:, d] = np.isin(nodes * dof + d, fixed).astype(np.int64)
    fe.add_dirichlet_boundary_condition(node_ids=nodes, dofs=mask, rhs=0.0)
    load = np.nonzero(wl["rhs"])[0]
    lnodes = np.unique(load // dof)
    forces = wl["rhs"].reshape(-1, dof)[lnodes]
    fe.add_point_forces(forces=forces, node_ids=lnodes)
    prob = MinimumCompliance(fe, filt, E_mul=[1.0], void=void, penalty=penalty,
                             volume_fraction=[vf], heavyside=False)
    return mesh, kern, fe, prob


def mbb_trajectory():
    """Config-1 MBB half-beam, 50 OC iterations with the reference direct solver."""
    wl = workloads.mbb2d(120, 40)
    _, _, fe, prob = _simp_setup(wl, lambda m, k: SPSOLVE(k), 1.5, 0.5)
    t = time.time()
    oc = OC(prob, move=0.2)
    f = [float(prob.f())]
    change = []
    for _ in range(50):
        oc.iter()
        f.append(float(prob.f()))
        change.append(float(oc.change))
    print(f"mbb: {time.time()-t:.1f}s f0={f[0]!r} f1={f[1]!r} f50={f[-1]!r}")
    save("mbb", f=np.array(f), change=np.array(change), x50=np.array(prob.get_desvars()),
         rhs=np.array(fe.rhs), cons=np.nonzero(fe.kernel.constraints)[0])
    return f


def pgd_goldens():
    """PGD (reference defaults, conjugate directions) on the config-1 MBB half-beam for 30
    iterations with the direct solver, the step size it chose at every iteration, and the
    reference's projection onto the volume constraint on stand-alone cases."""
    from pyFANTOM.Optimizers.CPU.PGD import PGD
    wl = workloads.mbb2d(120, 40)
    _, _, fe, prob = _simp_setup(wl, lambda m, k: SPSOLVE(k), 1.5, 0.5)
    t = time.time()
    x0 = np.array(prob.get_desvars())
    pgd = PGD(prob)
    out = {"x0": x0, "x_init": np.array(prob.get_desvars())}
    alphas = []
    orig = pgd.alpha

    def rec(*a):
        r = orig(*a)
        alphas.append(float(r[0]))
        return r

    pgd.alpha = rec
    f, change, change_f = [], [], []
    for it in range(30):
        pgd.iter()
        f.append(float(pgd.last_f))
        change.append(float(pgd.change))
        change_f.append(float(pgd.change_f))
        if it in (0, 1, 9, 29):
            out[f"x{it + 1}"] = np.array(prob.get_desvars())
    out.update(f=np.array(f), change=np.array(change), change_f=np.array(change_f), alpha=np.array(alphas),
               f_final=np.array(float(prob.f())))
    print(f"pgd: {time.time() - t:.1f}s f1={f[0]!r} f30={f[-1]!r}")
    # stand-alone projections: x_new = clip(xs + l dg, 0, 1) with the bisected l
    rng = np.random.default_rng(13)
    for tag, n, vf, lo, hi in [("p1", 4000, 0.4, -0.3, 1.4), ("p2", 2500, 0.25, 0.0, 1.0), ("p3", 3000, 0.6, -0.1, 0.5)]:
        xs = rng.uniform(lo, hi, n)
        dg = np.full(n, 1.0 / n)
        fake = _FixedProblem(np.clip(xs, 0, 1), np.zeros(n), vf)
        fake.dg = dg
        q = PGD.__new__(PGD)
        q.problem, q.is_independent, q.m, q.bounds, q.tol_B = fake, True, 1, (0, 1.0), 1e-8
        out[f"{tag}_xs"] = xs
        out[f"{tag}_vf"] = np.array(vf)
        out[f"{tag}_xnew"] = np.array(q.project_to_feasible(xs.copy(), xs.copy(), dg))
    save("pgd", **out)
    return f


class _FixedMultiProblem(_FixedProblem):
    """_FixedProblem with one volume constraint per material block (dg of shape (m, m ne),
    row i equal to 1/ne on block i, as MinimumCompliance builds it for m materials)."""

    def __init__(self, x, vf, m):
        super().__init__(x, np.zeros_like(x), np.asarray(vf, dtype=np.float64))
        ne = x.size // m
        self.dg = np.zeros((m, x.size))
        for i in range(m):
            self.dg[i, i * ne:(i + 1) * ne] = 1.0 / ne
        self._m = m

    def m(self):
        return self._m

    def g(self, rho=None):
        r = self.x if rho is None else rho
        return (self.dg @ r.reshape(-1, 1)).reshape(-1) - self.vf


def pgd_multi_goldens():
    """PGD with one volume constraint per material: the reference's projection
    (project_to_feasible, the independent-constraints branch with m > 1) on stand-alone
    cases, and 10 PGD iterations of the 2-material MBB half-beam (48x16, direct solve)."""
    from pyFANTOM.Optimizers.CPU.PGD import PGD
    rng = np.random.default_rng(29)
    out = {}
    # (tag, materials, elements per material, per-block (lo, hi) of the samples, volume fractions)
    cases = [("q1", 2, 3000, [(0.2, 1.3), (-0.2, 1.2)], [0.3, 0.5]),
             ("q2", 3, 2000, [(0.1, 1.1), (0.0, 0.3), (-0.3, 1.4)], [0.35, 0.5, 0.45]),
             ("q3", 2, 1500, [(0.0, 0.4), (-0.5, 0.5)], [0.6, 0.4])]
    for tag, m, ne, ranges, vf in cases:
        xs = np.concatenate([rng.uniform(lo, hi, ne) for lo, hi in ranges])
        fake = _FixedMultiProblem(np.clip(xs, 0, 1), vf, m)
        q = PGD.__new__(PGD)
        q.problem, q.is_independent, q.m, q.bounds, q.tol_B = fake, True, m, (0, 1.0), 1e-8
        out[f"{tag}_xs"] = xs
        out[f"{tag}_vf"] = np.array(vf)
        out[f"{tag}_xnew"] = np.array(q.project_to_feasible(xs.copy(), xs.copy(), fake.dg))
    wl = workloads.mbb2d(48, 16)
    _, _, fe, _ = _simp_setup(wl, lambda m, k: SPSOLVE(k), 1.5, 0.3)
    filt = StructuredFilter2D(fe.mesh, 1.5)
    prob = MinimumCompliance(fe, filt, E_mul=[1.0, 0.5], void=1e-9, penalty=3.0, volume_fraction=[0.15, 0.15],
                             heavyside=False)
    t = time.time()
    pgd = PGD(prob)  # initialises the design (uniform minimum volume fraction) and projects it
    out["mbb_x_init"] = np.array(prob.get_desvars())
    alphas = []
    orig = pgd.alpha

    def rec(*a):
        r = orig(*a)
        alphas.append(float(r[0]))
        return r

    pgd.alpha = rec
    f = []
    for it in range(10):
        pgd.iter()
        f.append(float(pgd.last_f))
        if it in (0, 1, 9):
            out[f"mbb_x{it + 1}"] = np.array(prob.get_desvars())
    out.update(mbb_f=np.array(f), mbb_alpha=np.array(alphas), mbb_g10=np.array(prob.g()))
    print(f"pgd multi-material: {time.time() - t:.1f}s f1={f[0]!r} f10={f[-1]!r}")
    save("pgd_multi", **out)


def sensitivity_goldens():
    """Compliance and its filtered sensitivity on a small bridge (direct solve)."""
    wl = workloads.bridge3d(12, 6, 6, seed=3)
    _, kern, fe, prob = _simp_setup(wl, lambda m, k: SPSOLVE(k), 2.5, 0.2)
    x = wl["x"]
    prob.set_desvars(x.copy())
    U = np.array(prob.FE.solve(prob.penalize(prob.filter.dot(x)))[0])
    save("sensitivity", x=x, f=np.array(prob.f()), df=np.array(prob.nabla_f()), U=U,
         rhs=np.array(fe.rhs), cons=np.nonzero(kern.constraints)[0], nel=np.array(wl["nel"]))


def solve_goldens():
    """Small cantilever: reference MultiGrid (CPU) and direct solve."""
    wl = workloads.cantilever3d(16, 8, 8, seed=0)
    out = {}
    for tag, fac in {"mg": lambda m, k: MultiGrid(m, k, maxiter=500, tol=1e-10, n_smooth=2, omega=0.6,
                                                    n_level=2, cycle="V"),
                     "direct": lambda m, k: SPSOLVE(k)}.items():
        _, kern, fe, _ = _simp_setup(wl, fac, 2.0, 0.3)
        U, res = fe.solve(wl["E"])
        out[f"{tag}_U"] = np.array(U)
        out[f"{tag}_res"] = np.array(res)
        out[f"{tag}_compliance"] = np.array(fe.rhs @ U)
    out["E"] = wl["E"]
    out["rhs"] = wl["rhs"]
    save("solve16", **out)


def odd_goldens():
    """2D grids with odd element counts, where every coarse grid floors nel / 2
    (core/CPU/_mgm.py, as core/CUDA/_mgm.py:24-27): restriction / prolongation, the Galerkin
    levels 1 and 2 with Dirichlet rows, and a MultiGrid solve of an MBB beam whose 3 coarse
    levels are 15x5 -> 7x2 -> 3x1 (at odd sizes the prolongation is not R^T, and the
    reference's PCG stagnates near 1e-3; the solve is recorded as it comes out) and one
    V-cycle on its hierarchy."""
    rng = np.random.default_rng(2024)
    out = {}
    for tag, nel in [("a", (7, 5)), ("b", (9, 6)), ("c", (6, 3))]:
        nel_a = np.array(nel, dtype=np.int32)
        nf = int(np.prod(nel_a + 1))
        nc = int(np.prod(nel_a // 2 + 1))
        vf = rng.standard_normal(nf * 2)
        vc = rng.standard_normal(nc * 2)
        out[f"{tag}_nel"] = nel_a
        out[f"{tag}_vf"] = vf
        out[f"{tag}_vc"] = vc
        out[f"{tag}_restricted"] = np.array(apply_restriction(vf, nel_a, 2))
        out[f"{tag}_prolonged"] = np.array(apply_prolongation(vc, nel_a, 2))
        mesh = StructuredMesh2D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        kern = StructuredStiffnessKernel(mesh)
        E = rng.uniform(1e-3, 1.0, mesh.elements.shape[0])
        kern.set_rho(E)
        x0 = np.where(mesh.nodes[:, 0] == 0)[0]
        cons = np.unique(np.concatenate([(x0[:, None] * 2 + np.arange(2)).reshape(-1),
                                         rng.choice(mesh.nodes.shape[0] * 2, size=3, replace=False)]))
        kern.add_constraints(cons)
        A1 = get_restricted_l0(mesh, kern)
        A2 = get_restricted_l1p(A1, mesh.nel // 2, 2)
        out[f"{tag}_E"] = E
        out[f"{tag}_cons"] = cons
        out[f"{tag}_A1"] = A1.toarray()
        out[f"{tag}_A2"] = A2.toarray()
    wl = workloads.mbb2d(30, 10)
    fac = lambda m, k: MultiGrid(m, k, maxiter=500, tol=1e-10, n_smooth=2, omega=0.6, n_level=3, cycle="V")  # noqa: E731
    _, kern, fe, _ = _simp_setup(wl, fac, 1.5, 0.5)
    U, res = fe.solve(wl["E"])
    out["mbb_U"] = np.array(U)
    out["mbb_res"] = np.array(res)
    out["mbb_E"] = wl["E"]
    # one V-cycle from a zero guess with level-0 Jacobi weight 0.45 (the reference's own
    # _multi_grid on the hierarchy the solve built)
    r = rng.standard_normal(np.array(fe.rhs).shape[0])
    r[np.nonzero(kern.constraints)[0]] = 0.0
    solver = fe.solver
    solver.matrix_free = False
    solver._setup()
    solver.coarse_solve = solver._coarse_solver(solver.levels[-1][0])
    solver.omega = 0.45
    out["mbb_r"] = r
    out["mbb_z"] = np.array(solver._multi_grid(np.zeros_like(r), r.copy(), 0))
    save("odd2d", **out)


def wcycle_goldens():
    """The lower-case 'w' cycle (solvers/CPU/_solvers.py _multi_grid, the second coarse
    correction at the levels in w_level): one cycle from a zero guess with level-0 Jacobi
    weight 0.45 for three w_level sets on a 16x8x8 cantilever (3 coarse levels), and
    MultiGrid solves with cycle='w' there and on a 32x16 MBB beam."""
    rng = np.random.default_rng(4242)
    out = {}
    wl = workloads.cantilever3d(16, 8, 8, seed=0)
    for tag, wlev in [("w0", [0]), ("w1", [1]), ("w01", [0, 1])]:
        fac = lambda m, k, wlev=wlev: MultiGrid(m, k, maxiter=500, tol=1e-10, n_smooth=2, omega=0.6,  # noqa: E731
                                                n_level=3, cycle="w", w_level=wlev)
        _, kern, fe, _ = _simp_setup(wl, fac, 2.0, 0.3)
        U, res = fe.solve(wl["E"])
        out[f"{tag}_U"] = np.array(U)
        out[f"{tag}_res"] = np.array(res)
        solver = fe.solver
        r = rng.standard_normal(np.array(fe.rhs).shape[0])
        r[np.nonzero(kern.constraints)[0]] = 0.0
        solver.matrix_free = False
        solver._setup()
        solver.coarse_solve = solver._coarse_solver(solver.levels[-1][0])
        solver.omega = 0.45
        out[f"{tag}_r"] = r
        out[f"{tag}_z"] = np.array(solver._multi_grid(np.zeros_like(r), r.copy(), 0))
    out["E"] = wl["E"]
    out["rhs"] = wl["rhs"]
    wl2 = workloads.mbb2d(32, 16)
    fac = lambda m, k: MultiGrid(m, k, maxiter=500, tol=1e-10, n_smooth=2, omega=0.6, n_level=3,  # noqa: E731
                                 cycle="w", w_level=1)
    _, kern, fe, _ = _simp_setup(wl2, fac, 1.5, 0.5)
    U, res = fe.solve(wl2["E"])
    out["mbb_U"] = np.array(U)
    out["mbb_res"] = np.array(res)
    out["mbb_E"] = wl2["E"]
    save("wcycle", **out)


def cg_goldens():
    """Textbook CG iterates: the reference's own CG loop (solvers/CPU/_solvers.py:111-139)
    run from x0 = 0 with rtol = 0 (never stops early), so that after maxiter = N it returns
    exactly the N-th iterate; the same iterates as cupyx cg, which the CUDA CG solver calls
    (solvers/CUDA/_solvers.py:114-127), from the same start."""
    out = {}
    for tag, wl, n_its in [("3d", workloads.cantilever3d(8, 4, 4, seed=3), (1, 7, 40)),
                           ("2d", workloads.mbb2d(16, 8), (1, 9, 60))]:
        _, kern, fe, _ = _simp_setup(wl, lambda m, k: SPSOLVE(k), 1.5, 0.5)
        kern.set_rho(wl["E"])
        rhs = np.array(fe.rhs)
        out[f"{tag}_nel"] = np.array(wl["nel"])
        out[f"{tag}_E"] = wl["E"]
        out[f"{tag}_rhs"] = rhs
        out[f"{tag}_cons"] = np.nonzero(kern.constraints)[0]
        out[f"{tag}_its"] = np.array(n_its)
        for n in n_its:
            x, _ = ref_cg(kern, rhs, x0=np.zeros_like(rhs), rtol=0.0, maxiter=n)
            out[f"{tag}_x{n}"] = np.array(x)
    save("cg", **out)


def big_solve():
    wl = workloads.cantilever3d(96, 48, 48, seed=0)
    fac = lambda m, k: MultiGrid(m, k, maxiter=1000, tol=1e-8, n_smooth=2, omega=0.6, n_level=4, cycle="V")
    _, kern, fe, _ = _simp_setup(wl, fac, 2.0, 0.3)
    t = time.time()
    U, res = fe.solve(wl["E"])
    dt = time.time() - t
    r = fe.rhs - kern.dot(U)
    true_res = float(np.linalg.norm(r) / np.linalg.norm(fe.rhs))
    c = float(fe.rhs @ U)
    print(f"config2 solve {dt:.1f}s compliance={c!r} true_res={true_res:.3e}")
    return dict(compliance=c, true_rel_res=true_res, seconds=dt, threads=os.cpu_count())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    ap.add_argument("--only", default=None, help="run one generator (e.g. pgd)")
    args = ap.parse_args()
    if args.only:
        globals()[f"{args.only}_goldens"]()
        return
    k0_goldens()
    operator_goldens()
    transfer_goldens()
    filter_goldens()
    oc_goldens()
    penalize_goldens()
    sensitivity_goldens()
    solve_goldens()
    cg_goldens()
    odd_goldens()
    f = mbb_trajectory()
    pgd_goldens()
    multimaterial_goldens()
    ka_path = os.path.join(HERE, "known_answers.json")
    ka = json.load(open(ka_path)) if os.path.exists(ka_path) else {}
    ka["mbb_120x40"] = {"f_init": f[0], "f_iter1": f[1], "f_iter50": f[50]}
    if args.big:
        ka["cantilever_96x48x48"] = big_solve()
    json.dump(ka, open(ka_path, "w"), indent=1)
    print("wrote known_answers.json")


if __name__ == "__main__":
    main()
