"""GPU: every kernel through the C ABI against the reference goldens and the oracle.

Tolerances: FP64 element operators 1e-12 relative (different but exact summation order),
FP32 matvec 2e-5 relative to the largest entry, integer / bisection work exact.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel, unit_K0
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from pyfantom_b200 import _lib
    _lib.require_cuda()
    return _lib


def T(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def N(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


class Op:
    def __init__(self, lib, nel, K0=None):
        self.lib = lib
        self.nel = tuple(int(v) for v in nel)
        self.dim = len(self.nel)
        self.grid = lib.make_grid(self.nel)
        K0 = unit_K0(self.dim) if K0 is None else K0
        self.K0 = np.ascontiguousarray(K0)
        self.h = ctypes.c_void_p()
        lib.check(lib.load().pf_op_create(ctypes.byref(self.grid), self.K0.ctypes.data, ctypes.byref(self.h)))
        self.n_nodes = int(np.prod(np.array(self.nel) + 1))
        self.ndof = self.n_nodes * self.dim

    def mask(self, cons):
        con = torch.zeros(self.ndof, dtype=torch.uint8, device="cuda")
        if cons is not None and len(cons):
            con[T(cons, torch.int64)] = 1
        m = torch.empty(self.n_nodes, dtype=torch.uint8, device="cuda")
        self.lib.check(self.lib.load().pf_pack_mask(self.h, self.lib.ptr(con), self.lib.ptr(m), self.lib.stream()))
        return m

    def matvec(self, E, u, cons=None, fp32=False):
        L = self.lib
        m = self.mask(cons) if cons is not None else None
        dt = torch.float32 if fp32 else torch.float64
        Et, ut = T(E, dt), T(u, dt)
        y = torch.full_like(ut, float("nan"))
        f = L.load().pf_matvec_f32 if fp32 else L.load().pf_matvec_f64
        L.check(f(self.h, L.ptr(Et), L.ptr(ut), L.ptr(m), L.ptr(y), L.stream()))
        return N(y)

    def diag(self, E, cons=None):
        L = self.lib
        m = self.mask(cons) if cons is not None else None
        d = torch.full((self.ndof,), float("nan"), dtype=torch.float64, device="cuda")
        Et = T(E)
        L.check(L.load().pf_diagonal_f64(self.h, L.ptr(Et), L.ptr(m), L.ptr(d), L.stream()))
        return N(d)

    def sens(self, U):
        L = self.lib
        dk = torch.full((int(np.prod(self.nel)),), float("nan"), dtype=torch.float64, device="cuda")
        Ut = T(U)
        L.check(L.load().pf_sensitivity_f64(self.h, L.ptr(Ut), L.ptr(dk), L.stream()))
        return N(dk)

    def __del__(self):
        if self.h.value:
            self.lib.load().pf_op_destroy(self.h)


@pytest.mark.parametrize("tag", ["3d", "3d_odd", "2d", "2d_odd"])
def test_matvec_diag_sens_golden(lib, golden, tag):
    g = golden("operators")
    op = Op(lib, g[tag + "_nel"])
    E, u, cons = g[tag + "_E"], g[tag + "_u"], g[tag + "_cons"]
    assert rel(op.matvec(E, u), g[tag + "_y_free"]) < 1e-12
    assert rel(op.matvec(E, u, cons), g[tag + "_y_con"]) < 1e-12
    assert rel(op.diag(E), g[tag + "_diag_free"]) < 1e-13
    assert rel(op.diag(E, cons), g[tag + "_diag_con"]) < 1e-13
    assert rel(op.sens(u), g[tag + "_dk"]) < 1e-12


@pytest.mark.parametrize("nel", [(1, 1, 1), (2, 3, 1), (40, 9, 33), (17, 70, 64), (12, 8, 31), (7, 5, 95),
                                 (64, 32, 32), (3, 2), (65, 33), (128, 1)])
def test_matvec_vs_oracle_shapes(lib, nel):
    """Tile edges: nz around multiples of 31, tiny and ragged grids, x-chunk boundaries."""
    rng = np.random.default_rng(sum(nel))
    op = Op(lib, nel)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(op.ndof)
    cons = rng.choice(op.ndof, size=max(1, op.ndof // 7), replace=False)
    K0 = op.K0
    assert rel(op.matvec(E, u), O.matvec(nel, K0, E, u)) < 1e-12
    assert rel(op.matvec(E, u, cons), O.matvec(nel, K0, E, u, cons)) < 1e-12
    y32 = op.matvec(E.astype(np.float32), u.astype(np.float32), cons, fp32=True)
    assert rel(y32, O.matvec(nel, K0, E.astype(np.float32), u.astype(np.float32), cons)) < 2e-5


@pytest.mark.parametrize("nel", [(3, 6, 29), (5, 13, 30), (70, 11, 59), (9, 22, 89), (130, 3, 3), (4, 12, 1)])
def test_matvec_march_tile_edges(lib, nel):
    """The x-march's own tiling: 30 owned node columns per warp (nz = 30, 31, 60, 90), 7
    (FP64) and 11 (FP32) owned node rows per block (ny = 7, 12, 14, 23), and x chunks of
    whatever length the wave model picks (nx = 4 .. 131), with constraints on a tenth of the
    DOFs, FP64 and FP32 against the oracle."""
    rng = np.random.default_rng(sum(nel) + 7)
    op = Op(lib, nel)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(op.ndof)
    cons = rng.choice(op.ndof, size=max(1, op.ndof // 10), replace=False)
    assert rel(op.matvec(E, u, cons), O.matvec(nel, op.K0, E, u, cons)) < 1e-12
    E32, u32 = E.astype(np.float32), u.astype(np.float32)
    assert rel(op.matvec(E32, u32, cons, fp32=True), O.matvec(nel, op.K0, E32, u32, cons)) < 2e-5


@pytest.mark.parametrize("nel", [(96, 48, 48), (64, 64, 64), (48, 96, 40)])
def test_matvec_large_and_repeatable(lib, nel):
    """Full-size grids (many blocks per SM, every tile and chunk edge) in FP64 and FP32, and
    bitwise run-to-run equality over repeated launches (catches shared-memory races)."""
    rng = np.random.default_rng(99)
    op = Op(lib, nel)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(op.ndof)
    cons = np.arange(0, 3 * (nel[2] + 1) * (nel[0] + 1), 1)  # the y = 0 face region, all DOFs
    ref = O.matvec(nel, op.K0, E, u, cons)
    y0 = op.matvec(E, u, cons)
    assert rel(y0, ref) < 1e-12
    for _ in range(10):
        assert np.array_equal(op.matvec(E, u, cons), y0)
    y32 = op.matvec(E.astype(np.float32), u.astype(np.float32), cons, fp32=True)
    ref32 = O.matvec(nel, op.K0, E.astype(np.float32), u.astype(np.float32), cons)
    assert rel(y32, ref32) < 2e-5
    for _ in range(10):
        assert np.array_equal(op.matvec(E.astype(np.float32), u.astype(np.float32), cons, fp32=True), y32)


def test_matvec_anisotropic_element(lib):
    K0 = unit_K0(3, nu=0.25, h=(1.0, 0.5, 2.0))
    nel = (6, 10, 4)
    rng = np.random.default_rng(5)
    op = Op(lib, nel, K0)
    E = rng.uniform(0.1, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(op.ndof)
    assert rel(op.matvec(E, u), O.matvec(nel, K0, E, u)) < 1e-12


def _walsh_T():
    cx, cy, cz = [0, 1, 1, 0, 0, 1, 1, 0], [0, 0, 1, 1, 0, 0, 1, 1], [0, 0, 0, 0, 1, 1, 1, 1]
    T = np.zeros((24, 24))
    for m in range(8):
        for l in range(8):
            s = 1
            for a, pos in enumerate((cx[l], cy[l], cz[l])):
                if (m >> a) & 1:
                    s *= 1 if pos else -1
            for c in range(3):
                T[m * 3 + c, l * 3 + c] = s
    return T


@pytest.mark.parametrize("kind", ["cube", "box", "dense"])
def test_matvec_element_operator_variants(lib, kind):
    """The three element-operator code paths: cube elements (7 coefficients), isotropic
    boxes (33 nonzero coefficients) and a reflection-symmetric K0 outside that pattern
    (dense class blocks), each in FP64 and FP32 against the oracle."""
    if kind == "cube":
        K0 = unit_K0(3)
    elif kind == "box":
        K0 = unit_K0(3, nu=0.25, h=(1.0, 0.5, 2.0))
    else:  # add a term coupling the x translations: class 1, row/column 0 becomes nonzero
        Tm = _walsh_T()
        dB = np.zeros((24, 24))
        dB[0, 0] = 0.01
        K0 = unit_K0(3) + Tm.T @ dB @ Tm
    nel = (20, 9, 37)
    rng = np.random.default_rng(11)
    op = Op(lib, nel, K0)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(op.ndof)
    cons = rng.choice(op.ndof, size=op.ndof // 9, replace=False)
    assert rel(op.matvec(E, u, cons), O.matvec(nel, K0, E, u, cons)) < 1e-12
    y32 = op.matvec(E.astype(np.float32), u.astype(np.float32), cons, fp32=True)
    assert rel(y32, O.matvec(nel, K0, E.astype(np.float32), u.astype(np.float32), cons)) < 2e-5


def test_matvec_symmetric_and_deterministic(lib):
    nel = (24, 12, 20)
    rng = np.random.default_rng(7)
    op = Op(lib, nel)
    E = rng.uniform(1e-3, 1, int(np.prod(nel)))
    u, v = rng.standard_normal(op.ndof), rng.standard_normal(op.ndof)
    cons = np.arange(0, op.ndof, 11)
    Ku, Kv = op.matvec(E, u, cons), op.matvec(E, v, cons)
    assert abs(Ku @ v - u @ Kv) < 1e-12 * abs(Ku @ v)
    assert np.array_equal(Ku, op.matvec(E, u, cons))  # run-to-run bitwise reproducible


def test_reject_asymmetric_k0(lib):
    K0 = unit_K0(3)
    K0[0, 1] += 1e-3
    g = lib.make_grid((2, 2, 2))
    h = ctypes.c_void_p()
    K0 = np.ascontiguousarray(K0)
    assert lib.load().pf_op_create(ctypes.byref(g), K0.ctypes.data, ctypes.byref(h)) == lib.PF_BAD_ARG


@pytest.mark.parametrize("tag", ["3d", "2d"])
def test_transfers_golden(lib, golden, tag):
    g = golden("transfers")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    grid = lib.make_grid(nel)
    vf, vc = T(g[tag + "_vf"]), T(g[tag + "_vc"])
    oc = torch.empty(O.n_nodes(O.coarse_nel(nel)) * len(nel), dtype=torch.float64, device="cuda")
    of = torch.empty(O.n_nodes(nel) * len(nel), dtype=torch.float64, device="cuda")
    L = lib.load()
    lib.check(L.pf_restrict_f64(ctypes.byref(grid), lib.ptr(vf), lib.ptr(oc), lib.stream()))
    lib.check(L.pf_prolong_f64(ctypes.byref(grid), lib.ptr(vc), lib.ptr(of), lib.stream()))
    assert rel(N(oc), g[tag + "_restricted"]) < 1e-15
    assert rel(N(of), g[tag + "_prolonged"]) < 1e-15


@pytest.mark.parametrize("nel", [(5, 4, 3), (7, 6, 9), (8, 4, 6), (2, 3, 2), (9, 5), (6, 7)])
def test_transfers_odd_and_even_sizes(lib, nel):
    """Restriction and prolongation (the 3D one by 2x2x2 cells of fine nodes) on grids with
    odd element counts, where the last fine node of an odd axis has a single parent, against
    the oracle (pinned to the reference on odd 2D grids)."""
    rng = np.random.default_rng(sum(nel))
    grid = lib.make_grid(nel)
    dim = len(nel)
    vf = rng.standard_normal(O.n_nodes(nel) * dim)
    vc = rng.standard_normal(O.n_nodes(O.coarse_nel(nel)) * dim)
    oc = torch.empty(vc.size, dtype=torch.float64, device="cuda")
    of = torch.empty(vf.size, dtype=torch.float64, device="cuda")
    vft, vct = T(vf), T(vc)
    L = lib.load()
    lib.check(L.pf_restrict_f64(ctypes.byref(grid), lib.ptr(vft), lib.ptr(oc), lib.stream()))
    lib.check(L.pf_prolong_f64(ctypes.byref(grid), lib.ptr(vct), lib.ptr(of), lib.stream()))
    assert rel(N(oc), O.restrict(nel, vf)) < 1e-15
    assert rel(N(of), O.prolong(nel, vc)) < 1e-15


def _soa_to_blocks(A, nn, dim):
    nb = 27 if dim == 3 else 9
    return A.reshape(nb, dim, dim, nn).transpose(3, 0, 1, 2)


@pytest.mark.parametrize("tag", ["3d", "2d"])
def test_galerkin_golden(lib, golden, tag):
    g = golden("transfers")
    nel = tuple(int(v) for v in g["gal" + tag + "_nel"])
    dim = len(nel)
    op = Op(lib, nel)
    m = op.mask(g["gal" + tag + "_cons"])
    c1 = O.coarse_nel(nel)
    c2 = O.coarse_nel(c1)
    g1, g2 = lib.make_grid(c1), lib.make_grid(c2)
    L = lib.load()
    A1 = torch.empty(int(L.pf_stencil_size(ctypes.byref(g1))), dtype=torch.float64, device="cuda")
    A2 = torch.empty(int(L.pf_stencil_size(ctypes.byref(g2))), dtype=torch.float64, device="cuda")
    Et = T(g["gal" + tag + "_E"])
    lib.check(L.pf_galerkin_l0_f64(op.h, lib.ptr(Et), lib.ptr(m), lib.ptr(A1), lib.stream()))
    lib.check(L.pf_galerkin_l1p_f64(ctypes.byref(g1), lib.ptr(A1), lib.ptr(A2), lib.stream()))
    B1 = _soa_to_blocks(N(A1), O.n_nodes(c1), dim)
    B2 = _soa_to_blocks(N(A2), O.n_nodes(c2), dim)
    assert rel(O.stencil_to_dense(c1, B1), g["gal" + tag + "_A1"]) < 1e-13
    assert rel(O.stencil_to_dense(c2, B2), g["gal" + tag + "_A2"]) < 1e-13


@pytest.mark.parametrize("nel", [(8, 4, 12), (16, 8, 8), (12, 20), (32, 64, 16)])
def test_galerkin_and_stencil_vs_oracle(lib, nel):
    rng = np.random.default_rng(11)
    dim = len(nel)
    op = Op(lib, nel)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    wl_cons = np.concatenate([np.arange(0, (nel[2] + 1 if dim == 3 else 1) * dim),  # a face strip at x = 0
                              rng.choice(op.ndof, size=op.ndof // 50 + 1, replace=False)])
    m = op.mask(wl_cons)
    c1 = O.coarse_nel(nel)
    g1 = lib.make_grid(c1)
    L = lib.load()
    A1 = torch.empty(int(L.pf_stencil_size(ctypes.byref(g1))), dtype=torch.float64, device="cuda")
    Et = T(E)
    lib.check(L.pf_galerkin_l0_f64(op.h, lib.ptr(Et), lib.ptr(m), lib.ptr(A1), lib.stream()))
    ref1 = O.galerkin_l0(nel, op.K0, E, wl_cons)
    B1 = _soa_to_blocks(N(A1), O.n_nodes(c1), dim)
    assert rel(B1, ref1) < 1e-13
    u = rng.standard_normal(O.n_nodes(c1) * dim)
    y = torch.empty(len(u), dtype=torch.float64, device="cuda")
    ut = T(u)
    lib.check(L.pf_stencil_matvec_f64(ctypes.byref(g1), lib.ptr(A1), lib.ptr(ut), lib.ptr(y), lib.stream()))
    assert rel(N(y), O.stencil_matvec(c1, ref1, u)) < 1e-13
    if all(v % 4 == 0 for v in nel):
        c2 = O.coarse_nel(c1)
        g2 = lib.make_grid(c2)
        A2 = torch.empty(int(L.pf_stencil_size(ctypes.byref(g2))), dtype=torch.float64, device="cuda")
        lib.check(L.pf_galerkin_l1p_f64(ctypes.byref(g1), lib.ptr(A1), lib.ptr(A2), lib.stream()))
        assert rel(_soa_to_blocks(N(A2), O.n_nodes(c2), dim), O.galerkin_l1p(c1, ref1)) < 1e-13


def _filter(lib, nel, w, off):
    grid = lib.make_grid(nel)
    h = ctypes.c_void_p()
    lib.check(lib.load().pf_filter_create(ctypes.byref(grid), len(w), np.ascontiguousarray(off, dtype=np.int32).ctypes.data,
                                          np.ascontiguousarray(w).ctypes.data, ctypes.byref(h)))
    return h


@pytest.mark.parametrize("tag", ["3d_r2", "3d_r25", "3d_aniso", "2d_r15", "2d_r3"])
def test_filter_golden(lib, golden, tag):
    g = golden("filters")
    nel = tuple(int(v) for v in g[tag + "_nel"])
    w, off = g[tag + "_weights"], g[tag + "_offsets"]
    h = _filter(lib, nel, w, off)
    L = lib.load()
    n = int(np.prod(nel))
    v = T(g[tag + "_v"])
    y, z, nrm = (torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3))
    lib.check(L.pf_filter_fwd_f64(h, lib.ptr(v), lib.ptr(y), lib.stream()))
    lib.check(L.pf_filter_adj_f64(h, lib.ptr(v), lib.ptr(z), lib.stream()))
    lib.check(L.pf_filter_normalizer_f64(h, lib.ptr(nrm), lib.stream()))
    assert rel(N(y), g[tag + "_fwd"]) < 1e-14
    assert rel(N(z), g[tag + "_adj"]) < 1e-14
    assert rel(N(nrm), g[tag + "_normalizer"]) < 1e-14
    L.pf_filter_destroy(h)


@pytest.mark.parametrize("tag", ["plain", "heavy", "emul"])
def test_penalize_golden(lib, golden, tag):
    from pyfantom_b200.Problem import penalize_device, simp_params
    g = golden("penalize")
    p = {"plain": simp_params(3.0, 1e-9, 1.0, 2.0, 0.5, False), "heavy": simp_params(3.0, 1e-9, 1.0, 4.0, 0.4, True),
         "emul": simp_params(2.5, 1e-6, 2.0, 2.0, 0.5, False)}[tag]
    E, dE = penalize_device(T(g["rho"]), p, True, True)
    assert rel(N(E), g[tag + "_E"]) < 1e-13
    assert rel(N(dE), g[tag + "_dE"]) < 1e-13


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_oc_golden(lib, golden, tag):
    g = golden("oc")
    x = T(g[tag + "_x"])
    n = x.numel()
    L = lib.load()
    work = torch.empty(int(L.pf_oc_workspace_size(n)), dtype=torch.float64, device="cuda")
    xn = torch.empty_like(x)
    out = (ctypes.c_double * 3)()
    dg = torch.full_like(x, 1.0 / n)
    dft = T(g[tag + "_df"])
    lib.check(L.pf_oc_update_f64(n, lib.ptr(x), lib.ptr(dft), lib.ptr(dg), float(g[tag + "_vf"]),
                                 float(g[tag + "_move"]), lib.ptr(xn), lib.ptr(work), out, lib.stream()))
    ref, steps = O.oc_update(g[tag + "_x"], g[tag + "_df"], 1.0 / n, float(g[tag + "_vf"]), float(g[tag + "_move"]))
    assert int(out[2]) == steps
    # the constraint sums differ only in summation order from the reference's
    assert np.abs(N(xn) - g[tag + "_xnew"]).max() < 1e-9
    assert abs(out[0] - np.linalg.norm(g[tag + "_x"] - ref)) < 1e-9


def test_dot(lib):
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal(1_000_003), rng.standard_normal(1_000_003)
    L = lib.load()
    work = torch.empty(int(L.pf_dot_workspace_size(a.size)), dtype=torch.float64, device="cuda")
    res = torch.empty(1, dtype=torch.float64, device="cuda")
    at, bt = T(a), T(b)
    lib.check(L.pf_dot_f64(a.size, lib.ptr(at), lib.ptr(bt), lib.ptr(res), lib.ptr(work), lib.stream()))
    assert abs(N(res)[0] - a @ b) < 1e-10 * np.abs(a * b).sum()


def _bf16_round(E):
    """E rounded to BF16 (round to nearest even), back as float64."""
    return torch.as_tensor(E, dtype=torch.float64).to(torch.bfloat16).to(torch.float64).numpy()


@pytest.mark.parametrize("nel", [(16, 8, 8), (40, 9, 33), (7, 5, 95), (65, 33)])
def test_matvec_bf16_element_scales(lib, nel):
    """FP32 matvec reading BF16 element scales: equal to the oracle's matvec with E rounded to
    BF16 (the only approximation is the storage of E) to FP32 rounding, 2e-5; the BF16
    rounding itself moves the product by at most 2^-8 relative to the FP64-E one."""
    rng = np.random.default_rng(sum(nel) + 3)
    op = Op(lib, nel)
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel)))
    u = rng.standard_normal(op.ndof).astype(np.float32)
    cons = rng.choice(op.ndof, size=max(1, op.ndof // 9), replace=False)
    L = lib
    Eb = torch.as_tensor(E, device="cuda").to(torch.bfloat16)
    ut = T(u, torch.float32)
    y = torch.full_like(ut, float("nan"))
    m = op.mask(cons)
    L.check(L.load().pf_matvec_f32_bf16(op.h, L.ptr(Eb), L.ptr(ut), L.ptr(m), L.ptr(y), L.stream()))
    got = N(y)
    assert rel(got, O.matvec(nel, op.K0, _bf16_round(E), u.astype(np.float64), cons)) < 2e-5
    assert rel(got, O.matvec(nel, op.K0, E, u.astype(np.float64), cons)) < 2 ** -8


def test_guess_select_picks_lower_energy(lib):
    """pf_cnn_guess_select_f64 on a small SPD system: the chosen guess is the energy-optimal
    multiple of the candidate with the lower energy -(x.f)^2 / (2 x.Kx)."""
    L = lib.load()
    rng = np.random.default_rng(5)
    n = 3000
    d = rng.uniform(1.0, 2.0, n)
    f = rng.standard_normal(n)
    u = f / d  # exact solution of the diagonal system K = diag(d)
    for xa, xb in [(u + 0.1 * rng.standard_normal(n), rng.standard_normal(n)),
                   (rng.standard_normal(n), 2.0 * u + 0.01 * rng.standard_normal(n)),
                   (np.zeros(n), u)]:
        ta, tb, tf = T(xa), T(xb), T(f)
        ka, kb = T(d * xa), T(d * xb)
        out = torch.empty_like(ta)
        work = torch.empty(int(L.pf_cnn_guess_select_workspace()), dtype=torch.float64, device="cuda")
        lib.check(L.pf_cnn_guess_select_f64(n, lib.ptr(ta), lib.ptr(ka), lib.ptr(tb), lib.ptr(kb), lib.ptr(tf),
                                            lib.ptr(out), lib.ptr(work), lib.stream()))

        def energy(x):
            q = x @ (d * x)
            return -0.5 * (x @ f) ** 2 / q if q > 0 else 0.0
        best = xb if energy(xb) < energy(xa) else xa
        q = best @ (d * best)
        want = (best @ f) / q * best if q > 0 else np.zeros(n)
        assert rel(N(out), want) < 1e-12
        assert N(work)[-3] == (1.0 if best is xb else 0.0)


@pytest.mark.parametrize("nel", [(5, 13, 61), (7, 12, 62), (9, 3, 63), (4, 23, 124), (70, 11, 125), (3, 2, 1),
                                 (13, 22, 186), (40, 12, 60)])
@pytest.mark.parametrize("variant", [0, 1])
def test_matvec_fp32_variants_tile_edges(lib, nel, variant):
    """Both FP32 fine matvecs of cube elements (variant 0: one element per thread; variant 1:
    two elements per thread in packed FP32, 62 owned node columns per warp and 11 owned node
    rows per block) on grids around their tile edges (nz + 1 = 62, 63, 64, 125, 126,
    187), with constraints on a tenth of the DOFs, against the oracle, and bitwise
    repeatable."""
    rng = np.random.default_rng(sum(nel) + 17 * variant)
    op = Op(lib, nel)
    lib.check(lib.load().pf_op_set_variant(op.h, variant))
    E = rng.uniform(1e-3, 1.0, int(np.prod(nel))).astype(np.float32)
    u = rng.standard_normal(op.ndof).astype(np.float32)
    cons = rng.choice(op.ndof, size=max(1, op.ndof // 10), replace=False)
    ref = O.matvec(nel, op.K0, E, u, cons)
    y = op.matvec(E, u, cons, fp32=True)
    assert rel(y, ref) < 2e-5
    assert rel(op.matvec(E, u, None, fp32=True), O.matvec(nel, op.K0, E, u)) < 2e-5
    assert np.array_equal(op.matvec(E, u, cons, fp32=True), y)


@pytest.mark.parametrize("variant", [0, 1])
def test_vcycle_fp32_variants_match(lib, variant):
    """The mixed-precision V-cycle (Jacobi, residual and correction epilogues of the FP32
    fine matvec) with either FP32 kernel agrees with the FP64 V-cycle to FP32 accuracy."""
    from pyfantom_b200 import workloads
    from pyfantom_b200.CUDA import MultiGrid, StructuredMesh3D, StructuredStiffnessKernel
    from pyfantom_b200.physics import LinearElasticity
    nel = (32, 16, 64)
    wl = workloads.cantilever3d(*nel)
    out = {}
    for prec in ("fp64", "mixed"):
        mesh = StructuredMesh3D(*nel, *nel, physics=LinearElasticity(E=1.0, nu=0.3))
        kern = StructuredStiffnessKernel(mesh)
        lib.check(lib.load().pf_op_set_variant(kern._op, variant))
        kern.add_constraints(torch.as_tensor(wl["fixed_dofs"], device="cuda"))
        kern.set_rho(torch.as_tensor(wl["E"], device="cuda"))
        sol = MultiGrid(mesh, kern, maxiter=100, tol=1e-8, n_smooth=2, omega=0.6, n_level=3, precision=prec)
        sol.setup()
        r = np.random.default_rng(1).standard_normal(kern.shape[0])
        r[wl["fixed_dofs"]] = 0.0
        out[prec] = sol.vcycle(torch.as_tensor(r, device="cuda"), omega=0.45).cpu().numpy()
    assert rel(out["mixed"], out["fp64"]) < 1e-4
