"""GPU: the element-level operator of multigrid level 1 against the assembled Galerkin
stencil (the library's own and the oracle's).

Level 1 is A1 = R (Z K Z + I - Z) P (reference mgm.cu:247-447); the element-level operator
applies it from the fine densities, with explicit matrices only for coarse elements that
touch a constraint.  It must equal the stencil A1 on every grid and constraint set: 1e-12
relative to the largest entry in FP64 (same sums in another order), 2e-5 in FP32 (the
V-cycle precision of the mixed forms).  Constraint sets: a clamped face (cantilever), two
pinned lines (bridge), and random single DOFs everywhere (every coarse element dirty or
next to one, which exercises the assignment of shared coefficient pairs to one element).
"""
import numpy as np
import pytest
import torch

from conftest import rel, unit_K0
from oracle import oracle as O
from pyfantom_b200 import workloads

pytestmark = pytest.mark.gpu


def _solver(nel, E, cons, n_level, precision="fp64", coarse_op="element", K0=None):
    from pyfantom_b200.CUDA import MultiGrid, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    if K0 is not None:
        mesh.K_single_host = np.ascontiguousarray(K0)
    kern = StructuredStiffnessKernel(mesh)
    if cons is not None and len(cons):
        kern.add_constraints(torch.as_tensor(cons, device="cuda"))
    kern.set_rho(torch.as_tensor(E, device="cuda"))
    sol = MultiGrid(mesh, kern, maxiter=200, tol=1e-8, n_smooth=2, omega=0.6, n_level=n_level,
                    precision=precision, coarse_op=coarse_op)
    sol.setup()
    return sol, kern


def _cases():
    rng = np.random.default_rng(11)
    out = []
    # level-1 z extents 2 .. 70: one z-tile of the x-march (30 owned node columns), two (62) and
    # three (70, the last partial)
    for nel in [(8, 4, 4), (16, 8, 12), (12, 4, 64), (4, 64, 4), (24, 16, 124), (60, 8, 8), (8, 6, 140)]:
        n_nodes = int(np.prod(np.array(nel) + 1))
        out.append((nel, "cantilever", workloads.cantilever3d(*nel)["fixed_dofs"]))
        out.append((nel, "bridge", workloads.bridge3d(*nel)["fixed_dofs"]))
        out.append((nel, "random", np.unique(rng.choice(3 * n_nodes, size=max(4, n_nodes // 6), replace=False))))
    out.append(((16, 8, 8), "none", np.array([], dtype=np.int64)))
    return out


@pytest.mark.parametrize("nel,kind,cons", _cases(), ids=lambda v: str(v) if not isinstance(v, np.ndarray) else "")
def test_level1_element_operator_equals_stencil(nel, kind, cons):
    rng = np.random.default_rng(sum(nel) + len(kind))
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    sol, kern = _solver(nel, E, cons, 2)
    elem, dirty = sol.level_info()
    assert elem
    if kind == "none":
        assert dirty == 0
    cnel = tuple(n // 2 for n in nel)
    nc = int(np.prod(np.array(cnel) + 1)) * 3
    u = rng.standard_normal(nc)
    y = sol.level_matvec(1, torch.as_tensor(u, device="cuda")).cpu().numpy()
    A1 = O.galerkin_l0(nel, unit_K0(3), E, cons if len(cons) else None)
    yo = O.stencil_matvec(cnel, A1, u)
    assert rel(y, yo) < 1e-12
    ref, _ = _solver(nel, E, cons, 2, coarse_op="stencil")
    assert not ref.level_info()[0]
    ys = ref.level_matvec(1, torch.as_tensor(u, device="cuda")).cpu().numpy()
    assert rel(y, ys) < 1e-12
    # FP32 V-cycle operator
    s32, _ = _solver(nel, E, cons, 2, precision="mixed")
    y32 = s32.level_matvec(1, torch.as_tensor(u, dtype=torch.float32, device="cuda")).cpu().numpy()
    assert rel(y32, yo) < 2e-5


@pytest.mark.parametrize("kind", ["cantilever", "bridge", "random"])
def test_level1_row_accuracy_at_simp_contrast(kind):
    """SIMP contrast (solid 1, void 1e-9, void everywhere next to the constraints): every
    row of the operator to 1e-5 (FP32) and 1e-12 (FP64) of that row's |A1| |u|, the accuracy
    an assembled FP32 stencil has.  The identity rows of constrained fine DOFs are O(1) where
    the void stiffness is O(1e-9); mixed into one Walsh-basis element matrix they would leave
    the void rows of the FP32 operator with errors of order one."""
    nel = (16, 8, 12)
    rng = np.random.default_rng(17)
    wl = workloads.cantilever3d(*nel) if kind != "bridge" else workloads.bridge3d(*nel)
    cons = wl["fixed_dofs"]
    if kind == "random":
        n_nodes = int(np.prod(np.array(nel) + 1))
        cons = np.unique(rng.choice(3 * n_nodes, size=n_nodes // 6, replace=False))
    ex = np.repeat(np.arange(nel[0]), nel[1] * nel[2])  # element order: x slowest
    E = np.where(rng.uniform(size=int(np.prod(nel))) < 0.5, 1e-9, 1.0)
    if kind != "random":
        E[ex <= 1] = 1e-9  # void at and next to the clamped face / supports
        E[ex >= nel[0] - 2] = 1e-9
    cnel = tuple(n // 2 for n in nel)
    nc = int(np.prod(np.array(cnel) + 1)) * 3
    A1 = O.galerkin_l0(nel, unit_K0(3), E, cons)
    u = rng.standard_normal(nc).astype(np.float32).astype(np.float64)
    yo = O.stencil_matvec(cnel, A1, u)
    scale = O.stencil_matvec(cnel, np.abs(A1), np.abs(u))
    s64, _ = _solver(nel, E, cons, 2)
    assert s64.level_info()[0] and s64.level_info()[1] > 0
    y64 = s64.level_matvec(1, torch.as_tensor(u, device="cuda")).cpu().numpy()
    assert np.max(np.abs(y64 - yo) / scale) < 1e-12
    s32, _ = _solver(nel, E, cons, 2, precision="mixed")
    y32 = s32.level_matvec(1, torch.as_tensor(u, dtype=torch.float32, device="cuda")).cpu().numpy()
    assert np.max(np.abs(y32 - yo) / scale) < 1e-5


def test_level1_repeated_setup_and_growing_dirty_set():
    """Setups with new densities and a larger constraint set (the dirty storage grows and
    the solver's captured iterations are rebuilt): the operator follows each change."""
    nel = (16, 8, 8)
    rng = np.random.default_rng(3)
    from pyfantom_b200.CUDA import MultiGrid, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
    kern = StructuredStiffnessKernel(mesh)
    wl = workloads.cantilever3d(*nel)
    kern.add_constraints(torch.as_tensor(wl["fixed_dofs"], device="cuda"))
    sol = MultiGrid(mesh, kern, maxiter=300, tol=1e-10, n_smooth=2, omega=0.6, n_level=2, coarse_op="element")
    rhs = torch.as_tensor(wl["rhs"], device="cuda")
    cons = np.array(wl["fixed_dofs"])
    for step in range(4):
        E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
        if step == 2:
            extra = rng.choice(kern.shape[0], size=300, replace=False)
            cons = np.unique(np.concatenate([cons, extra]))
            kern.add_constraints(torch.as_tensor(extra, device="cuda"))
        U, res = sol.solve(rhs, rho=torch.as_tensor(E, device="cuda"), use_last=False)
        assert sol.last_info["status"] == "PF_OK" and res < 1e-10
        assert sol.level_info()[0]
        u = rng.standard_normal(int(np.prod(np.array(nel) // 2 + 1)) * 3)
        y = sol.level_matvec(1, torch.as_tensor(u, device="cuda")).cpu().numpy()
        A1 = O.galerkin_l0(nel, unit_K0(3), E, cons)
        assert rel(y, O.stencil_matvec(tuple(n // 2 for n in nel), A1, u)) < 1e-12
        xo, ito, _, _ = O.mgcg_solve(nel, unit_K0(3), E, cons, wl["rhs"], n_level=2, tol=1e-10)
        assert abs(sol.last_info["iterations"] - ito) <= 1
        assert rel(U.cpu().numpy(), xo) < 1e-8


CX = [0, 1, 1, 0, 0, 1, 1, 0]
CY = [0, 0, 1, 1, 0, 0, 1, 1]
CZ = [0, 0, 0, 0, 1, 1, 1, 1]


def _reflection(axis):
    """24x24 matrix of the element's reflection along `axis`: corners swap along that axis
    (reference local corner order) and the displacement component along it changes sign."""
    pos = [(CX[l], CY[l], CZ[l]) for l in range(8)]
    R = np.zeros((24, 24))
    for l in range(8):
        p = list(pos[l])
        p[axis] = 1 - p[axis]
        l2 = pos.index(tuple(p))
        for c in range(3):
            R[l2 * 3 + c, l * 3 + c] = -1.0 if c == axis else 1.0
    return R


def test_level1_falls_back_to_stencil_without_isotropic_structure():
    """A K0 that keeps the reflection symmetry the fine operator needs but not the isotropic
    box pattern: level 1 uses its stencil, and the V-cycle still equals the oracle's."""
    K0 = unit_K0(3)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((24, 24)) * 0.01
    X = X @ X.T
    Rs = [np.eye(24)]
    for a in range(3):
        Rs = Rs + [R @ _reflection(a) for R in Rs]
    K1 = K0 + sum(R @ X @ R.T for R in Rs) / len(Rs)
    nel = (16, 8, 8)
    wl = workloads.cantilever3d(*nel)
    sol, kern = _solver(nel, wl["E"], wl["fixed_dofs"], 2, K0=K1)
    assert sol.level_info() == (False, 0)
    r = rng.standard_normal(kern.shape[0])
    r[wl["fixed_dofs"]] = 0.0
    z = sol.vcycle(torch.as_tensor(r, device="cuda"), omega=0.45).cpu().numpy()
    zr = O.mg_vcycle(nel, K1, wl["E"], wl["fixed_dofs"], r, n_level=2, n_smooth=2, omega=0.45)
    assert rel(z, zr) < 1e-10


@pytest.mark.parametrize("nel,kind", [((32, 16, 16), "cantilever"), ((40, 22, 26), "bridge"), ((34, 17, 21), "cantilever"),
                                      ((32, 16, 16), "none")])
def test_levels_2_and_3_equal_oracle_galerkin_chain(nel, kind):
    """Levels 2 and 3 of the hierarchy (built by the separable Galerkin product: one pass per
    axis) against the oracle's Galerkin chain R A P from the level-1 stencil, as operators,
    on even and odd grids with and without constraints: 1e-12 relative (same sums in
    another order)."""
    rng = np.random.default_rng(sum(nel))
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    wl = workloads.bridge3d(*nel) if kind == "bridge" else workloads.cantilever3d(*nel)
    cons = wl["fixed_dofs"] if kind != "none" else np.array([], dtype=np.int64)
    sol, kern = _solver(nel, E, cons, 4)
    A = O.galerkin_l0(nel, unit_K0(3), E, cons if len(cons) else None)
    cnel = O.coarse_nel(nel)
    for level in (2, 3):
        A = O.galerkin_l1p(cnel, A)
        cnel = O.coarse_nel(cnel)
        u = rng.standard_normal(O.n_nodes(cnel) * 3)
        y = sol.level_matvec(level, torch.as_tensor(u, device="cuda")).cpu().numpy()
        assert rel(y, O.stencil_matvec(cnel, A, u)) < 1e-12, level
