"""ctypes front-end of the CPU oracle (oracle/pf_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, by ``__graft_entry__.smoke()`` as the checker
and by ``bench.py`` for the CPU-baseline / reference arm.  The library under
``pyfantom_b200`` never imports it.

Every array argument is a numpy array (float64 / int32 / uint8); results are returned
as new numpy arrays.  Grid conventions are those of the reference structured mesh
(pyFANTOM/core/CUDA/Kernels/_geom.py:23-49); coarse operators are dense block
stencils ``A[node, nb, dof, dof]`` with ``nb = (dx+1) + 3(dy+1) [+ 9(dz+1)]``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpf_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_bp = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> str:
    """Compile pf_oracle.c with the system gcc (OpenMP) if needed; returns the .so path."""
    src = os.path.join(_HERE, "pf_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-s", "-C", _HERE, "CC=gcc"], check=True, env=env)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        V = None
        sigs = {
            "or_matvec": (V, [ctypes.c_int, _ip, _dp, _dp, _dp, _bp, _dp]),
            "or_diagonal": (V, [ctypes.c_int, _ip, _dp, _dp, _bp, _dp]),
            "or_process_dk": (V, [ctypes.c_int, _ip, _dp, _dp, _dp]),
            "or_restrict": (V, [ctypes.c_int, _ip, _dp, _dp]),
            "or_prolong": (V, [ctypes.c_int, _ip, _dp, _dp]),
            "or_galerkin_l0": (V, [ctypes.c_int, _ip, _dp, _dp, _bp, _dp]),
            "or_galerkin_l1p": (V, [ctypes.c_int, _ip, _dp, _dp]),
            "or_stencil_matvec": (V, [ctypes.c_int, _ip, _dp, _dp, _dp]),
            "or_stencil_to_dense": (V, [ctypes.c_int, _ip, _dp, _dp]),
            "or_cholesky": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_double, _dp]),
            "or_cholesky_solve": (V, [ctypes.c_int, _dp, _dp, _dp]),
            "or_mgcg_solve": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             _dp, _dp, _bp, _dp, _dp, ctypes.c_int, _dp, _ip]),
            "or_mgcg_solve_timed": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                   _dp, _dp, _bp, _dp, _dp, ctypes.c_int, _dp, _ip, _dp]),
            "or_mgcg_solve_deflated": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                      _dp, _dp, _bp, _dp, _dp, ctypes.c_int, _dp, _dp, _ip]),
            "or_cg_solve": (ctypes.c_int, [ctypes.c_int, _ip, _dp, _dp, _bp, _dp, _dp, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_int, _dp]),
            "or_mg_vcycle": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, _dp, _dp, _bp, _dp, _dp]),
            "or_mg_cycle": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_uint, _dp, _dp, _bp, _dp, _dp]),
            "or_mgcg_solve_w": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                               _dp, _dp, _bp, _dp, _dp, ctypes.c_int, ctypes.c_uint, _dp, _ip]),
            "or_mgcg_solve_ex": (ctypes.c_int, [ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                _dp, _dp, _bp, _dp, _dp, ctypes.c_int, _dp, ctypes.c_uint,
                                                ctypes.c_double, _dp, _ip]),
            "or_filter_normalizer": (V, [ctypes.c_int, _ip, ctypes.c_int, _ip, _dp, _dp]),
            "or_filter_fwd": (V, [ctypes.c_int, _ip, ctypes.c_int, _ip, _dp, _dp, _dp]),
            "or_filter_adj": (V, [ctypes.c_int, _ip, ctypes.c_int, _ip, _dp, _dp, _dp, _dp]),
            "or_oc_update": (ctypes.c_int, [ctypes.c_long, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp]),
            "or_num_threads": (ctypes.c_int, []),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _con(con, ndof):
    if con is None:
        return None, None
    c = np.zeros(ndof, dtype=np.uint8)
    con = np.asarray(con)
    if con.dtype == bool and con.size == ndof:
        c[:] = con
    else:
        c[con.astype(np.int64)] = 1
    return c, c.ctypes.data_as(_bp)


def n_nodes(nel):
    return int(np.prod(np.asarray(nel) + 1))


def n_elem(nel):
    return int(np.prod(np.asarray(nel)))


def coarse_nel(nel):
    return tuple(int(n) // 2 for n in nel)


def matvec(nel, K0, w, u, con=None):
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ua, pu = _d(u)
    ca, pc = _con(con, nd)
    out = np.zeros(nd)
    lib().or_matvec(dim, pn, pK, pw, pu, pc, out.ctypes.data_as(_dp))
    return out


def diagonal(nel, K0, w, con=None):
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ca, pc = _con(con, nd)
    out = np.zeros(nd)
    lib().or_diagonal(dim, pn, pK, pw, pc, out.ctypes.data_as(_dp))
    return out


def process_dk(nel, K0, U):
    dim = len(nel)
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    Ua, pU = _d(U)
    out = np.zeros(n_elem(nel))
    lib().or_process_dk(dim, pn, pK, pU, out.ctypes.data_as(_dp))
    return out


def restrict(nel, vf):
    dim = len(nel)
    nel_a, pn = _i(nel)
    va, pv = _d(vf)
    out = np.zeros(n_nodes(coarse_nel(nel)) * dim)
    lib().or_restrict(dim, pn, pv, out.ctypes.data_as(_dp))
    return out


def prolong(nel, vc):
    dim = len(nel)
    nel_a, pn = _i(nel)
    va, pv = _d(vc)
    out = np.zeros(n_nodes(nel) * dim)
    lib().or_prolong(dim, pn, pv, out.ctypes.data_as(_dp))
    return out


def _nb(dim):
    return 27 if dim == 3 else 9


def galerkin_l0(nel, K0, w, con=None):
    """Level-1 block stencil from the fine operator (shape [n_coarse_nodes, nb, dof, dof])."""
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ca, pc = _con(con, nd)
    out = np.zeros((n_nodes(coarse_nel(nel)), _nb(dim), dim, dim))
    lib().or_galerkin_l0(dim, pn, pK, pw, pc, out.ctypes.data_as(_dp))
    return out


def galerkin_l1p(nel, A):
    """Next-level block stencil from the level-(nel) stencil ``A``."""
    dim = len(nel)
    nel_a, pn = _i(nel)
    Aa, pA = _d(A)
    out = np.zeros((n_nodes(coarse_nel(nel)), _nb(dim), dim, dim))
    lib().or_galerkin_l1p(dim, pn, pA, out.ctypes.data_as(_dp))
    return out


def stencil_matvec(nel, A, u):
    dim = len(nel)
    nel_a, pn = _i(nel)
    Aa, pA = _d(A)
    ua, pu = _d(u)
    out = np.zeros(n_nodes(nel) * dim)
    lib().or_stencil_matvec(dim, pn, pA, pu, out.ctypes.data_as(_dp))
    return out


def stencil_to_dense(nel, A):
    dim = len(nel)
    N = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    Aa, pA = _d(A)
    out = np.zeros((N, N))
    lib().or_stencil_to_dense(dim, pn, pA, out.ctypes.data_as(_dp))
    return out


def mgcg_solve(nel, K0, w, con, rhs, n_level=3, n_smooth=2, omega=0.6, min_omega=0.4, omega_boost=1.06,
               tol=1e-8, maxiter=1000, x0=None, deflation=None, w_level=(), fixed_omega=None):
    """MultiGrid-preconditioned CG with the reference CUDA semantics.  ``deflation``: a
    nodal field whose components span a deflation space of the PCG (the library's learned
    coarse-grid correction, pf_mg_set_deflation; no reference counterpart).  ``w_level``:
    the levels where the reference's lower-case 'w' cycle applies its second coarse
    correction (solvers/CUDA/_solvers.py:550-569); empty for the V-cycle.  ``fixed_omega``:
    a Jacobi weight kept through the solve instead of the reference's schedule (the
    library's option of the same name; no reference counterpart).

    Returns (x, iterations, relative recursive residual, status)."""
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ca, pc = _con(con, nd)
    ra, pr = _d(rhs)
    x = np.zeros(nd) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    res = ctypes.c_double(0.0)
    st = ctypes.c_int(0)
    if w_level or fixed_omega is not None:
        py = _d(deflation)[1] if deflation is not None else None
        it = lib().or_mgcg_solve_ex(dim, pn, n_level, n_smooth, omega, min_omega, omega_boost, tol, maxiter,
                                    pK, pw, pc, pr, x.ctypes.data_as(_dp), int(x0 is not None), py, _w_mask(w_level),
                                    float(fixed_omega or 0.0), ctypes.byref(res), ctypes.byref(st))
    elif deflation is not None:
        ya, py = _d(deflation)
        it = lib().or_mgcg_solve_deflated(dim, pn, n_level, n_smooth, omega, min_omega, omega_boost, tol, maxiter,
                                          pK, pw, pc, pr, x.ctypes.data_as(_dp), int(x0 is not None), py,
                                          ctypes.byref(res), ctypes.byref(st))
    else:
        it = lib().or_mgcg_solve(dim, pn, n_level, n_smooth, omega, min_omega, omega_boost, tol, maxiter,
                                 pK, pw, pc, pr, x.ctypes.data_as(_dp), int(x0 is not None),
                                 ctypes.byref(res), ctypes.byref(st))
    return x, int(it), float(res.value), int(st.value)


def mgcg_solve_timed(nel, K0, w, con, rhs, n_level=3, n_smooth=2, omega=0.6, min_omega=0.4, omega_boost=1.06,
                     tol=1e-8, maxiter=1000):
    """``mgcg_solve`` from x0 = 0 that also returns the wall-clock seconds of the hierarchy
    setup and of the PCG iterations: (x, iterations, residual, status, setup_s, iterate_s)."""
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ca, pc = _con(con, nd)
    ra, pr = _d(rhs)
    x = np.zeros(nd)
    res = ctypes.c_double(0.0)
    st = ctypes.c_int(0)
    t = np.zeros(2)
    it = lib().or_mgcg_solve_timed(dim, pn, n_level, n_smooth, omega, min_omega, omega_boost, tol, maxiter,
                                   pK, pw, pc, pr, x.ctypes.data_as(_dp), 0, ctypes.byref(res), ctypes.byref(st),
                                   t.ctypes.data_as(_dp))
    return x, int(it), float(res.value), int(st.value), float(t[0]), float(t[1])


def cg_solve(nel, K0, w, con, rhs, tol=1e-5, maxiter=1000, x0=None):
    """Unpreconditioned textbook CG (the cupyx ``cg`` the reference CG solver calls,
    solvers/CUDA/_solvers.py:114-127).  Returns (x, iterations, relative residual)."""
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ca, pc = _con(con, nd)
    ra, pr = _d(rhs)
    x = np.zeros(nd) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    res = ctypes.c_double(0.0)
    it = lib().or_cg_solve(dim, pn, pK, pw, pc, pr, x.ctypes.data_as(_dp), int(x0 is not None), tol, maxiter,
                           ctypes.byref(res))
    return x, int(it), float(res.value)


def _w_mask(w_level):
    m = 0
    for l in w_level:
        if not 0 <= int(l) < 32:
            raise ValueError(f"w_level {l} out of range")
        m |= 1 << int(l)
    return m


def mg_vcycle(nel, K0, w, con, r, n_level=3, n_smooth=2, omega=0.4, omega_boost=1.06, w_level=()):
    """One cycle z = M r from a zero guess (level-0 Jacobi weight ``omega``): the V-cycle,
    or with ``w_level`` the lower-case 'w' cycle (second coarse correction at those levels)."""
    dim = len(nel)
    nd = n_nodes(nel) * dim
    nel_a, pn = _i(nel)
    K0a, pK = _d(K0)
    wa, pw = _d(w)
    ca, pc = _con(con, nd)
    ra, pr = _d(r)
    z = np.zeros(nd)
    st = lib().or_mg_cycle(dim, pn, n_level, n_smooth, omega, omega_boost, _w_mask(w_level), pK, pw, pc, pr,
                           z.ctypes.data_as(_dp))
    if st:
        raise RuntimeError(f"coarse Cholesky failed at pivot {st}")
    return z


def filter_weights(nel, h, r_min):
    """Cone weights and integer offsets, restating geom/CUDA/_filters.py:65-98 (3D) and
    the 2D twin: offsets over [-ceil(r), ceil(r)]^dim (meshgrid 'ij' order), distances
    scaled by h/min(h), w = (r - d)/r kept where > 0, normalised to sum 1."""
    dim = len(nel)
    h = np.asarray(h, dtype=np.float64)
    scales = h / h.min()
    n = int(np.ceil(r_min))
    rng = np.arange(-n, n + 1, dtype=np.int32)
    grids = np.meshgrid(*([rng] * dim), indexing="ij")
    offsets = np.vstack([g.ravel() for g in grids]).T
    d = np.linalg.norm(offsets * scales[None], axis=1)
    w = (r_min - d) / r_min
    keep = w > 0
    offsets, w = offsets[keep], w[keep]
    w = w / w.sum()
    return w.astype(np.float64), offsets.astype(np.int32)


def filter_normalizer(nel, weights, offsets):
    dim = len(nel)
    nel_a, pn = _i(nel)
    wa, pw = _d(weights)
    oa, po = _i(offsets)
    out = np.zeros(n_elem(nel))
    lib().or_filter_normalizer(dim, pn, len(wa), po, pw, out.ctypes.data_as(_dp))
    return out


def filter_fwd(nel, weights, offsets, v):
    dim = len(nel)
    nel_a, pn = _i(nel)
    wa, pw = _d(weights)
    oa, po = _i(offsets)
    va, pv = _d(v)
    out = np.zeros(n_elem(nel))
    lib().or_filter_fwd(dim, pn, len(wa), po, pw, pv, out.ctypes.data_as(_dp))
    return out


def filter_adj(nel, weights, offsets, normalizer, v):
    dim = len(nel)
    nel_a, pn = _i(nel)
    wa, pw = _d(weights)
    oa, po = _i(offsets)
    na, pnm = _d(normalizer)
    va, pv = _d(v)
    out = np.zeros(n_elem(nel))
    lib().or_filter_adj(dim, pn, len(wa), po, pw, pnm, pv, out.ctypes.data_as(_dp))
    return out


def oc_update(x, df, dg, vf, move):
    """One OC step; returns (x_new, bisection steps)."""
    xa, px = _d(x)
    fa, pf = _d(df)
    ga, pg = _d(np.broadcast_to(np.asarray(dg, dtype=np.float64), xa.shape))
    out = np.zeros_like(xa)
    steps = lib().or_oc_update(len(xa), px, pf, pg, float(vf), float(move), out.ctypes.data_as(_dp))
    return out, int(steps)


def penalize_multi(rho, E_mul, penalty=3.0, void=1e-9, heavyside=False, beta=2.0, eta=0.5):
    """Multi-material SIMP law and its gradient (pyFANTOM/Problem/CPU/MinimumCompliance.py
    multi-material branches): rho [nel, nm] -> (E [nel], dE [nel, nm]) with a_i = H(rho_i)^p,
    E = max(sum_i E_mul_i a_i prod_{j != i} (1 - a_j), void) and its derivative."""
    rho = np.asarray(rho, np.float64)
    E_mul = np.asarray(E_mul, np.float64)
    nm = rho.shape[1]
    if heavyside:
        den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
        h = (np.tanh(beta * eta) + np.tanh(beta * (rho - eta))) / den
        dh = beta * (1 - np.tanh(beta * (rho - eta)) ** 2) / den
    else:
        h, dh = rho, np.ones_like(rho)
    a, da = h ** penalty, penalty * h ** (penalty - 1)
    b = 1.0 - a
    E = np.zeros(rho.shape[0])
    dE = np.zeros_like(rho)
    for i in range(nm):
        t = a[:, i].copy()
        for j in range(nm):
            if j != i:
                t *= b[:, j]
        E += E_mul[i] * t
    for k in range(nm):
        for i in range(nm):
            t = da[:, k].copy() if i == k else -da[:, k] * a[:, i]
            for j in range(nm):
                if j != i and j != k:
                    t *= b[:, j]
            dE[:, k] += E_mul[i] * t
        dE[:, k] *= dh[:, k]
    return np.maximum(E, void), dE


def pgd_project(xs, dg, vf, lo=0.0, hi=1.0, tol=1e-8):
    """The reference PGD projection for one volume constraint
    (pyFANTOM/Optimizers/CPU/PGD.py:144-170): clip(xs + l dg, lo, hi) with l bisected in
    [-1e12, 0] (midpoint rule, l2 = mid when dg.x - vf <= 0, else l1 = mid) until
    (l2 - l1) / (l2 + l1) <= tol; returns (x_new, l, steps)."""
    xs, dg = np.asarray(xs, np.float64), np.asarray(dg, np.float64)
    l1, l2 = 0.0, -1e12
    d = np.clip(xs + l1 * dg, lo, hi)
    if dg @ d - vf <= 0.0:
        return d, 0.0, 0
    steps, lm = 0, 0.0
    while (l2 - l1) / (l2 + l1) > tol:
        lm = (l1 + l2) / 2
        d = np.clip(xs + lm * dg, lo, hi)
        if dg @ d - vf <= 0.0:
            l2 = lm
        else:
            l1 = lm
        steps += 1
    return d, lm, steps


def pgd_project_multi(xs, dg, vf, lo=0.0, hi=1.0, tol=1e-8):
    """The reference PGD projection for m independent volume constraints, one per block of
    the design (pyFANTOM/Optimizers/CPU/PGD.py:146-170 with m > 1; MinimumCompliance's
    constraint rows are block-diagonal, Problem/CPU/MinimumCompliance.py:111-118).
    xs (m, ne): the design by block; dg (m, ne): row i of the constraint gradient on
    block i; vf (m,).  The m bisections run in lockstep: every sweep moves every shift to
    its midpoint, and the sweeps continue while ANY block's (l2 - l1) / (l2 + l1) exceeds
    tol (a block whose clip(xs) is feasible keeps l1 = 0, so its ratio stays 1 until l2
    underflows to zero, about 1100 sweeps).  When clip(xs) is feasible in every block the
    result is clip(xs).  Returns (x_new (m, ne), l (m,), sweeps)."""
    xs, dg = np.asarray(xs, np.float64), np.asarray(dg, np.float64)
    vf = np.asarray(vf, np.float64)
    m = xs.shape[0]
    d = np.clip(xs, lo, hi)
    if np.all(np.einsum("ij,ij->i", dg, d) - vf <= 0.0):
        return d, np.zeros(m), 0
    l1, l2 = np.zeros(m), np.full(m, -1e12)
    lm = np.zeros(m)
    sweeps = 0
    with np.errstate(invalid="ignore"):
        while np.any((l2 - l1) / (l2 + l1) > tol):
            lm = (l1 + l2) / 2
            d = np.clip(xs + lm[:, None] * dg, lo, hi)
            ok = np.einsum("ij,ij->i", dg, d) - vf <= 0.0
            l2 = np.where(ok, lm, l2)
            l1 = np.where(ok, l1, lm)
            sweeps += 1
    return d, lm, sweeps


def penalize(rho, penalty=3.0, void=1e-9, E_mul=1.0, heavyside=False, beta=2.0, eta=0.5):
    """SIMP law, Problem/CUDA/MinimumCompliance.py:305-324 (single material)."""
    rho = np.asarray(rho, dtype=np.float64)
    if heavyside:
        den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
        rho = (np.tanh(beta * eta) + np.tanh(beta * (rho - eta))) / den
    e = np.clip(rho ** penalty, void, 1.0) * E_mul
    return np.clip(e, void, None)


def penalize_grad(rho, penalty=3.0, E_mul=1.0, heavyside=False, beta=2.0, eta=0.5):
    """dE/drho without the clip term, Problem/CUDA/MinimumCompliance.py:351-367."""
    rho = np.asarray(rho, dtype=np.float64)
    if heavyside:
        den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
        rh = (np.tanh(beta * eta) + np.tanh(beta * (rho - eta))) / den
        df = penalty * rh ** (penalty - 1) * beta * (1 - np.tanh(beta * (rho - eta)) ** 2) / den
    else:
        df = penalty * rho ** (penalty - 1)
    return df * E_mul


def num_threads():
    return int(lib().or_num_threads())
