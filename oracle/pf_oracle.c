/*
 * pf_oracle.c -- CPU oracle for the structured SIMP / MGCG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C with OpenMP, the algorithms
 * of the reference pyFANTOM path (CUDA semantics) so that the CUDA library can be
 * checked against it and so that a CPU baseline can be timed.  The library never links
 * or calls it.  Each function cites the reference source it follows.  The restatement is
 * pinned against fixtures generated by running the reference's own CPU code
 * (tests/golden/make_golden.py).
 *
 * Conventions (reference pyFANTOM/core/CUDA/Kernels/_geom.py:23-49):
 *   3D node (i,j,k) -> k + nz*i + nz*nx*j ; element (i,j,k) -> i*nely*nelz + j*nelz + k
 *   2D node (i,j)   -> i + nx*j           ; element (i,j)   -> i*nely + j
 *   element corner l has offsets CX[l], CY[l], CZ[l]; DOF = node*dof + d.
 *   Constraint masks are one byte per DOF (1 = Dirichlet).
 *   Coarse operators are stored as dense block stencils A[node][nb][dof][dof] with
 *   nb = (dx+1) + 3*(dy+1) (+ 9*(dz+1) in 3D): the same 27 (9) blocks per row, in the same
 *   order, as the reference's padded CSR (mgm.cu:384-395, 81 / 18 entries per row).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const int CX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int CY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int CZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

typedef struct {
    int dim, dof, nc; /* nc = corners per element */
    int nel[3], nn[3];
    long n_nodes, n_elem;
} grid_t;

static grid_t mkgrid(int dim, const int* nel) {
    grid_t g;
    memset(&g, 0, sizeof(g));
    g.dim = dim;
    g.dof = dim;
    g.nc = dim == 3 ? 8 : 4;
    g.n_nodes = 1;
    g.n_elem = 1;
    for (int a = 0; a < 3; a++) {
        g.nel[a] = a < dim ? nel[a] : 0;
        g.nn[a] = a < dim ? nel[a] + 1 : 1;
        if (a < dim) {
            g.n_nodes *= g.nn[a];
            g.n_elem *= g.nel[a];
        }
    }
    return g;
}

static inline long node_id(const grid_t* g, int i, int j, int k) {
    if (g->dim == 3) return (long)k + (long)g->nn[2] * i + (long)g->nn[2] * g->nn[0] * j;
    return (long)i + (long)g->nn[0] * j;
}
static inline void node_ijk(const grid_t* g, long n, int* i, int* j, int* k) {
    if (g->dim == 3) {
        *k = (int)(n % g->nn[2]);
        long t = n / g->nn[2];
        *i = (int)(t % g->nn[0]);
        *j = (int)(t / g->nn[0]);
    } else {
        *i = (int)(n % g->nn[0]);
        *j = (int)(n / g->nn[0]);
        *k = 0;
    }
}
static inline long elem_id(const grid_t* g, int i, int j, int k) {
    if (g->dim == 3) return (long)i * g->nel[1] * g->nel[2] + (long)j * g->nel[2] + k;
    return (long)i * g->nel[1] + j;
}
static inline int elem_ok(const grid_t* g, int i, int j, int k) {
    if (i < 0 || j < 0 || i >= g->nel[0] || j >= g->nel[1]) return 0;
    if (g->dim == 3 && (k < 0 || k >= g->nel[2])) return 0;
    return 1;
}
static inline int node_ok(const grid_t* g, int i, int j, int k) {
    if (i < 0 || j < 0 || i >= g->nn[0] || j >= g->nn[1]) return 0;
    if (g->dim == 3 && (k < 0 || k >= g->nn[2])) return 0;
    return 1;
}
static inline int cz(const grid_t* g, int l) { return g->dim == 3 ? CZ[l] : 0; }

/* ------------------------------------------------------------------------------------
 * Stiffness matvec with Dirichlet identity rows, node-gather form.
 * Follows matvec.cu:45-98 (mat_vec_node_basis_parallel_wcon_cuda_kernel) and
 * core/CPU/_ops.py:332-368: out[c] = vec[c] at constrained DOFs; constrained columns are
 * skipped; out_i = sum_{e containing i} w_e * sum_l K0[row(i in e)][l] * vec[col l].
 * con may be NULL (no constraints: matvec.cu:1-43).
 * ---------------------------------------------------------------------------------- */
void or_matvec(int dim, const int* nel, const double* K0, const double* w, const double* vec,
               const uint8_t* con, double* out) {
    grid_t g = mkgrid(dim, nel);
    const int dof = g.dof, nd = g.nc * dof;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < g.n_nodes; n++) {
        int i, j, k;
        node_ijk(&g, n, &i, &j, &k);
        for (int d = 0; d < dof; d++) out[n * dof + d] = (con && con[n * dof + d]) ? vec[n * dof + d] : 0.0;
        for (int r = 0; r < g.nc; r++) { /* node n is corner r of element (i-CX[r], ...) */
            int ei = i - CX[r], ej = j - CY[r], ek = k - cz(&g, r);
            if (!elem_ok(&g, ei, ej, ek)) continue;
            double we = w[elem_id(&g, ei, ej, ek)];
            for (int d = 0; d < dof; d++) {
                if (con && con[n * dof + d]) continue;
                double val = 0.0;
                for (int l = 0; l < g.nc; l++) {
                    long m = node_id(&g, ei + CX[l], ej + CY[l], ek + cz(&g, l));
                    for (int dd = 0; dd < dof; dd++) {
                        if (con && con[m * dof + dd]) continue;
                        val += K0[(r * dof + d) * nd + l * dof + dd] * vec[m * dof + dd];
                    }
                }
                out[n * dof + d] += val * we;
            }
        }
    }
}

/* diag(K(w)) with 1 at constrained DOFs.  Follows diag.cu:1-47, core/CPU/_ops.py:45-75. */
void or_diagonal(int dim, const int* nel, const double* K0, const double* w, const uint8_t* con,
                 double* diag) {
    grid_t g = mkgrid(dim, nel);
    const int dof = g.dof, nd = g.nc * dof;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < g.n_nodes; n++) {
        int i, j, k;
        node_ijk(&g, n, &i, &j, &k);
        for (int d = 0; d < dof; d++) {
            if (con && con[n * dof + d]) {
                diag[n * dof + d] = 1.0;
                continue;
            }
            double s = 0.0;
            for (int r = 0; r < g.nc; r++) {
                int ei = i - CX[r], ej = j - CY[r], ek = k - cz(&g, r);
                if (!elem_ok(&g, ei, ej, ek)) continue;
                s += K0[(r * dof + d) * nd + r * dof + d] * w[elem_id(&g, ei, ej, ek)];
            }
            diag[n * dof + d] = s;
        }
    }
}

/* dk_e = -u_e^T K0 u_e.  Follows grad.cu:1-16 (process_dk_kernel_cuda), core/CPU/_ops.py:5-13. */
void or_process_dk(int dim, const int* nel, const double* K0, const double* U, double* dk) {
    grid_t g = mkgrid(dim, nel);
    const int dof = g.dof, nd = g.nc * dof;
#pragma omp parallel for schedule(static)
    for (long e = 0; e < g.n_elem; e++) {
        int i, j, k;
        if (dim == 3) {
            i = (int)(e / ((long)g.nel[1] * g.nel[2]));
            j = (int)((e / g.nel[2]) % g.nel[1]);
            k = (int)(e % g.nel[2]);
        } else {
            i = (int)(e / g.nel[1]);
            j = (int)(e % g.nel[1]);
            k = 0;
        }
        double ue[24];
        for (int l = 0; l < g.nc; l++) {
            long m = node_id(&g, i + CX[l], j + CY[l], k + cz(&g, l));
            for (int d = 0; d < dof; d++) ue[l * dof + d] = U[m * dof + d];
        }
        double out = 0.0;
        for (int a = 0; a < nd; a++) {
            double val = 0.0;
            for (int b = 0; b < nd; b++) val += K0[a * nd + b] * ue[b];
            out -= val * ue[a];
        }
        dk[e] = out;
    }
}

/* ------------------------------------------------------------------------------------
 * Grid transfers.  Restriction r_c = sum 0.5^{|d|_1} r_f / tw(c); prolongation
 * e_f = mean over parent coarse nodes of e_c / tw(c).  tw = product over axes of
 * (1.5 if the coarse node is on that axis' boundary else 2).
 * Follows mgm.cu:1-244 (restriction_3d/2d_kernel, prolongation_3d/2d_kernel).
 * nel is the FINE element count; the coarse grid has nel/2 elements (floor, as the
 * reference).
 * ---------------------------------------------------------------------------------- */
static double total_weight(const grid_t* gc, int i, int j, int k) {
    int b = 0;
    if (i == 0 || i == gc->nn[0] - 1) b++;
    if (j == 0 || j == gc->nn[1] - 1) b++;
    if (gc->dim == 3) {
        if (k == 0 || k == gc->nn[2] - 1) b++;
        return b == 3 ? 3.375 : b == 2 ? 4.5 : b == 1 ? 6.0 : 8.0;
    }
    return b == 2 ? 2.25 : b == 1 ? 3.0 : 4.0;
}
static double pow_half(int dist) { return dist == 0 ? 1.0 : dist == 1 ? 0.5 : dist == 2 ? 0.25 : 0.125; }

static grid_t coarse_of(const grid_t* gf) {
    int nc[3] = {gf->nel[0] / 2, gf->nel[1] / 2, gf->dim == 3 ? gf->nel[2] / 2 : 0};
    return mkgrid(gf->dim, nc);
}

void or_restrict(int dim, const int* nel, const double* vf, double* vc) {
    grid_t gf = mkgrid(dim, nel), gc = coarse_of(&gf);
    const int dof = gf.dof, kr = dim == 3 ? 1 : 0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < gc.n_nodes; c++) {
        int ic, jc, kc;
        node_ijk(&gc, c, &ic, &jc, &kc);
        double tw = total_weight(&gc, ic, jc, kc);
        for (int d = 0; d < dof; d++) {
            double value = 0.0;
            for (int di = -1; di <= 1; di++)
                for (int dj = -1; dj <= 1; dj++)
                    for (int dk = -kr; dk <= kr; dk++) {
                        int fi = 2 * ic + di, fj = 2 * jc + dj, fk = 2 * kc + dk;
                        if (!node_ok(&gf, fi, fj, fk)) continue;
                        value += pow_half(abs(di) + abs(dj) + abs(dk)) * vf[node_id(&gf, fi, fj, fk) * dof + d];
                    }
            vc[c * dof + d] = value / tw;
        }
    }
}

void or_prolong(int dim, const int* nel, const double* vc, double* vf) {
    grid_t gf = mkgrid(dim, nel), gc = coarse_of(&gf);
    const int dof = gf.dof;
#pragma omp parallel for schedule(static)
    for (long f = 0; f < gf.n_nodes; f++) {
        int i, j, k;
        node_ijk(&gf, f, &i, &j, &k);
        for (int d = 0; d < dof; d++) {
            double value = 0.0;
            int count = 0;
            for (int ci = i / 2; ci <= i / 2 + (i % 2); ci++) {
                if (ci >= gc.nn[0]) continue;
                for (int cj = j / 2; cj <= j / 2 + (j % 2); cj++) {
                    if (cj >= gc.nn[1]) continue;
                    int k0 = dim == 3 ? k / 2 : 0, k1 = dim == 3 ? k / 2 + (k % 2) : 0;
                    for (int ck = k0; ck <= k1; ck++) {
                        if (dim == 3 && ck >= gc.nn[2]) continue;
                        value += vc[node_id(&gc, ci, cj, ck) * dof + d] / total_weight(&gc, ci, cj, ck);
                        count++;
                    }
                }
            }
            vf[f * dof + d] = count > 0 ? value / count : 0.0;
        }
    }
}

/* ------------------------------------------------------------------------------------
 * Galerkin coarse operators.
 * or_galerkin_l0: level-1 operator R (Z K Z + I - Z) P from K0, w and the constraint
 * mask, per (coarse node, neighbour).  Follows mgm.cu:247-447 (get_target_vals,
 * get_restricted_3d_l0_nnz_based) and the 2D twins mgm.cu:592-740.
 * or_galerkin_l1p: level l+1 from the level-l block stencil.  Follows mgm.cu:449-590
 * (get_target_vals_l1p, get_restricted_3d_l1p_nnz_based).
 * Output blocks: A[(c*nb + o)*dof*dof + a*dof + b], o = (dx+1)+3(dy+1)+9(dz+1).
 * ---------------------------------------------------------------------------------- */
static int n_blocks(int dim) { return dim == 3 ? 27 : 9; }
static void nb_offsets(int dim, int o, int* dx, int* dy, int* dz) {
    *dx = o % 3 - 1;
    *dy = (o / 3) % 3 - 1;
    *dz = dim == 3 ? (o / 9) % 3 - 1 : 0;
}

void or_galerkin_l0(int dim, const int* nel, const double* K0, const double* w, const uint8_t* con,
                    double* A) {
    grid_t gf = mkgrid(dim, nel), gc = coarse_of(&gf);
    const int dof = gf.dof, nd = gf.nc * dof, NB = n_blocks(dim), kr = dim == 3 ? 1 : 0;
    memset(A, 0, sizeof(double) * gc.n_nodes * NB * dof * dof);
#pragma omp parallel for schedule(dynamic, 16)
    for (long c = 0; c < gc.n_nodes; c++) {
        int ic, jc, kc;
        node_ijk(&gc, c, &ic, &jc, &kc);
        double tw = total_weight(&gc, ic, jc, kc);
        for (int o = 0; o < NB; o++) {
            int ox, oy, oz;
            nb_offsets(dim, o, &ox, &oy, &oz);
            int ti = ic + ox, tj = jc + oy, tk = kc + oz;
            if (!node_ok(&gc, ti, tj, tk)) continue;
            double twt = total_weight(&gc, ti, tj, tk);
            int fti = 2 * ti, ftj = 2 * tj, ftk = 2 * tk;
            double* blk = A + (c * NB + o) * dof * dof;
            for (int di = -1; di <= 1; di++)
                for (int dj = -1; dj <= 1; dj++)
                    for (int dk = -kr; dk <= kr; dk++) {
                        int fi = 2 * ic + di, fj = 2 * jc + dj, fk = 2 * kc + dk;
                        if (!node_ok(&gf, fi, fj, fk)) continue;
                        double wgt = pow_half(abs(di) + abs(dj) + abs(dk));
                        long n = node_id(&gf, fi, fj, fk);
                        double vals[9] = {0};
                        /* identity rows of constrained DOFs (mgm.cu:261-288) */
                        for (int a = 0; a < dof; a++) {
                            if (!(con && con[n * dof + a])) continue;
                            int ddi = fi - fti, ddj = fj - ftj, ddk = fk - ftk;
                            if (ddi < -1 || ddi > 1 || ddj < -1 || ddj > 1 || ddk < -1 || ddk > 1) continue;
                            vals[a * dof + a] = pow_half(abs(ddi) + abs(ddj) + abs(ddk));
                        }
                        /* element contributions (mgm.cu:290-338) */
                        for (int r = 0; r < gf.nc; r++) {
                            int ei = fi - CX[r], ej = fj - CY[r], ek = fk - cz(&gf, r);
                            if (!elem_ok(&gf, ei, ej, ek)) continue;
                            double rho = w[elem_id(&gf, ei, ej, ek)];
                            for (int l = 0; l < gf.nc; l++) {
                                int mi = ei + CX[l], mj = ej + CY[l], mk = ek + cz(&gf, l);
                                int ddi = mi - fti, ddj = mj - ftj, ddk = mk - ftk;
                                if (ddi < -1 || ddi > 1 || ddj < -1 || ddj > 1 || ddk < -1 || ddk > 1) continue;
                                double wt = pow_half(abs(ddi) + abs(ddj) + abs(ddk));
                                long m = node_id(&gf, mi, mj, mk);
                                for (int a = 0; a < dof; a++) {
                                    if (con && con[n * dof + a]) continue;
                                    for (int b = 0; b < dof; b++) {
                                        if (con && con[m * dof + b]) continue;
                                        vals[a * dof + b] += K0[(r * dof + a) * nd + l * dof + b] * wt * rho;
                                    }
                                }
                            }
                        }
                        for (int a = 0; a < dof * dof; a++) blk[a] += wgt * vals[a] / tw / twt;
                    }
        }
    }
}

void or_galerkin_l1p(int dim, const int* nel, const double* Af, double* Ac) {
    grid_t gf = mkgrid(dim, nel), gc = coarse_of(&gf);
    const int dof = gf.dof, NB = n_blocks(dim), kr = dim == 3 ? 1 : 0, bs = dof * dof;
    memset(Ac, 0, sizeof(double) * gc.n_nodes * NB * bs);
#pragma omp parallel for schedule(dynamic, 16)
    for (long c = 0; c < gc.n_nodes; c++) {
        int ic, jc, kc;
        node_ijk(&gc, c, &ic, &jc, &kc);
        double tw = total_weight(&gc, ic, jc, kc);
        for (int o = 0; o < NB; o++) {
            int ox, oy, oz;
            nb_offsets(dim, o, &ox, &oy, &oz);
            int ti = ic + ox, tj = jc + oy, tk = kc + oz;
            if (!node_ok(&gc, ti, tj, tk)) continue;
            double twt = total_weight(&gc, ti, tj, tk);
            int fti = 2 * ti, ftj = 2 * tj, ftk = 2 * tk;
            double* blk = Ac + (c * NB + o) * bs;
            for (int di = -1; di <= 1; di++)
                for (int dj = -1; dj <= 1; dj++)
                    for (int dk = -kr; dk <= kr; dk++) {
                        int fi = 2 * ic + di, fj = 2 * jc + dj, fk = 2 * kc + dk;
                        if (!node_ok(&gf, fi, fj, fk)) continue;
                        double wgt = pow_half(abs(di) + abs(dj) + abs(dk));
                        long n = node_id(&gf, fi, fj, fk);
                        double vals[9] = {0};
                        for (int o2 = 0; o2 < NB; o2++) {
                            int px, py, pz;
                            nb_offsets(dim, o2, &px, &py, &pz);
                            int mi = fi + px, mj = fj + py, mk = fk + pz;
                            if (!node_ok(&gf, mi, mj, mk)) continue;
                            int ddi = mi - fti, ddj = mj - ftj, ddk = mk - ftk;
                            if (ddi < -1 || ddi > 1 || ddj < -1 || ddj > 1 || ddk < -1 || ddk > 1) continue;
                            double wt = pow_half(abs(ddi) + abs(ddj) + abs(ddk));
                            const double* src = Af + (n * NB + o2) * bs;
                            for (int a = 0; a < bs; a++) vals[a] += src[a] * wt;
                        }
                        for (int a = 0; a < bs; a++) blk[a] += wgt * vals[a] / tw / twt;
                    }
        }
    }
}

/* y = A u for a block stencil (CSR SpMV of the reference's padded CSR, _solvers.py:439). */
void or_stencil_matvec(int dim, const int* nel_of_level, const double* A, const double* u, double* y) {
    grid_t g = mkgrid(dim, nel_of_level);
    const int dof = g.dof, NB = n_blocks(dim), bs = dof * dof;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < g.n_nodes; n++) {
        int i, j, k;
        node_ijk(&g, n, &i, &j, &k);
        double acc[3] = {0, 0, 0};
        for (int o = 0; o < NB; o++) {
            int ox, oy, oz;
            nb_offsets(dim, o, &ox, &oy, &oz);
            if (!node_ok(&g, i + ox, j + oy, k + oz)) continue;
            long m = node_id(&g, i + ox, j + oy, k + oz);
            const double* blk = A + (n * NB + o) * bs;
            for (int a = 0; a < dof; a++)
                for (int b = 0; b < dof; b++) acc[a] += blk[a * dof + b] * u[m * dof + b];
        }
        for (int a = 0; a < dof; a++) y[n * dof + a] = acc[a];
    }
}

/* diagonal of a block stencil (csr_diagonal, diag.cu:149-160) */
void or_stencil_diagonal(int dim, const int* nel_of_level, const double* A, double* d) {
    grid_t g = mkgrid(dim, nel_of_level);
    const int dof = g.dof, NB = n_blocks(dim), bs = dof * dof, oc = NB / 2;
    for (long n = 0; n < g.n_nodes; n++)
        for (int a = 0; a < dof; a++) d[n * dof + a] = A[(n * NB + oc) * bs + a * dof + a];
}

/* ------------------------------------------------------------------------------------
 * Dense Cholesky of (A + beta I) (CHOLMOD cholesky(K, beta), _solvers.py:508-514) and
 * the triangular solves.  L is row-major lower; returns 0 or the failing pivot + 1.
 * ---------------------------------------------------------------------------------- */
int or_cholesky(int n, const double* A, double beta, double* L) {
    memcpy(L, A, sizeof(double) * n * n);
    for (int i = 0; i < n; i++) L[(long)i * n + i] += beta;
    for (int j = 0; j < n; j++) {
        double s = L[(long)j * n + j];
        for (int k = 0; k < j; k++) s -= L[(long)j * n + k] * L[(long)j * n + k];
        if (!(s > 0.0)) return j + 1;
        double ljj = sqrt(s);
        L[(long)j * n + j] = ljj;
#pragma omp parallel for schedule(static) if (n > 256)
        for (int i = j + 1; i < n; i++) {
            double t = L[(long)i * n + j];
            for (int k = 0; k < j; k++) t -= L[(long)i * n + k] * L[(long)j * n + k];
            L[(long)i * n + j] = t / ljj;
        }
    }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) L[(long)i * n + j] = 0.0;
    return 0;
}

void or_cholesky_solve(int n, const double* L, const double* b, double* x) {
    for (int i = 0; i < n; i++) {
        double s = b[i];
        for (int k = 0; k < i; k++) s -= L[(long)i * n + k] * x[k];
        x[i] = s / L[(long)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int k = i + 1; k < n; k++) s -= L[(long)k * n + i] * x[k];
        x[i] = s / L[(long)i * n + i];
    }
}

/* Dense matrix of a block stencil (the coarsest level, for the Cholesky). */
void or_stencil_to_dense(int dim, const int* nel_of_level, const double* A, double* M) {
    grid_t g = mkgrid(dim, nel_of_level);
    const int dof = g.dof, NB = n_blocks(dim), bs = dof * dof;
    long N = g.n_nodes * dof;
    memset(M, 0, sizeof(double) * N * N);
    for (long n = 0; n < g.n_nodes; n++) {
        int i, j, k;
        node_ijk(&g, n, &i, &j, &k);
        for (int o = 0; o < NB; o++) {
            int ox, oy, oz;
            nb_offsets(dim, o, &ox, &oy, &oz);
            if (!node_ok(&g, i + ox, j + oy, k + oz)) continue;
            long m = node_id(&g, i + ox, j + oy, k + oz);
            for (int a = 0; a < dof; a++)
                for (int b = 0; b < dof; b++) M[(n * dof + a) * N + m * dof + b] += A[(n * NB + o) * bs + a * dof + b];
        }
    }
}

/* ------------------------------------------------------------------------------------
 * MultiGrid-preconditioned CG with the reference CUDA semantics
 * (solvers/CUDA/_solvers.py:437-660):
 *   setup: D0 = 1/diag(K), level 1 = galerkin_l0, level l>=2 = galerkin_l1p, D = 1/diag,
 *          coarse = Cholesky(A_L + 1e-6 I);
 *   V-cycle(x=0, b, l): n_smooth Jacobi sweeps with omega*1.06^l, r = b - A x, restrict,
 *          recurse from zero, prolong, n_smooth Jacobi sweeps on A e = r from the
 *          prolonged e, x += e  (the 'W' default behaves as a V-cycle);
 *   the lower-case 'w' cycle (_solvers.py:550-569) repeats that coarse correction once
 *          more, from the updated x, at every level l in w_level (bit l of w_mask);
 *   PCG: omega starts at min_omega; after each iteration
 *          omega = min_omega + d_omega/2 * exp(-500 (clip(R, tol, 0.1) - tol))
 *          (or a fixed weight throughout: the library's fixed_omega option).
 * ---------------------------------------------------------------------------------- */
typedef struct {
    int dim, n_level, n_smooth;
    int nel[8][3];
    long ndof[8];
    const double* K0;
    const double* w;
    const uint8_t* con;
    double* A[8];   /* level >= 1 stencils */
    double* Dinv[8];
    double* Lc;     /* coarse Cholesky factor */
    double omega_boost;
    unsigned w_mask; /* levels that take the 'w' cycle's second coarse correction */
    double* tmp[8][5]; /* per level: 0 r, 1 b, 2 e, 3 Ax, 4 x */
} mg_t;

static void level_matvec(mg_t* m, int l, const double* u, double* y) {
    if (l == 0)
        or_matvec(m->dim, m->nel[0], m->K0, m->w, u, m->con, y);
    else
        or_stencil_matvec(m->dim, m->nel[l], m->A[l], u, y);
}

static void jacobi(mg_t* m, int l, double* x, const double* b, double omega, int x_is_zero) {
    long n = m->ndof[l];
    double* Ax = m->tmp[l][3];
    for (int s = 0; s < m->n_smooth; s++) {
        if (s == 0 && x_is_zero) {
#pragma omp parallel for
            for (long i = 0; i < n; i++) x[i] = omega * m->Dinv[l][i] * b[i];
            continue;
        }
        level_matvec(m, l, x, Ax);
#pragma omp parallel for
        for (long i = 0; i < n; i++) x[i] += omega * m->Dinv[l][i] * (b[i] - Ax[i]);
    }
}

static void vcycle(mg_t* m, int l, double* x, const double* b, double omega) {
    long n = m->ndof[l];
    if (l == m->n_level) {
        or_cholesky_solve((int)n, m->Lc, b, x);
        return;
    }
    double wl = omega * pow(m->omega_boost, l);
    memset(x, 0, sizeof(double) * n);
    jacobi(m, l, x, b, wl, 1);
    const int passes = ((m->w_mask >> l) & 1u) ? 2 : 1;
    for (int pass = 0; pass < passes; pass++) {
        double* r = m->tmp[l][0];
        double* Ax = m->tmp[l][3];
        level_matvec(m, l, x, Ax);
#pragma omp parallel for
        for (long i = 0; i < n; i++) r[i] = b[i] - Ax[i];
        double* rc = m->tmp[l + 1][1];
        double* ec = m->tmp[l + 1][4];
        or_restrict(m->dim, m->nel[l], r, rc);
        vcycle(m, l + 1, ec, rc, omega);
        double* e = m->tmp[l][2];
        or_prolong(m->dim, m->nel[l], ec, e);
        jacobi(m, l, e, r, wl, 0);
#pragma omp parallel for
        for (long i = 0; i < n; i++) x[i] += e[i];
    }
}

/* deterministic dot product: 64 fixed chunks summed in order (an OpenMP reduction
 * combines thread partials in arrival order, which varies from run to run) */
static double dot(long n, const double* a, const double* b) {
    enum { NCH = 64 };
    double part[NCH];
#pragma omp parallel for schedule(static)
    for (int c = 0; c < NCH; c++) {
        const long lo = n * c / NCH, hi = n * (c + 1) / NCH;
        double s = 0.0;
        for (long i = lo; i < hi; i++) s += a[i] * b[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int c = 0; c < NCH; c++) s += part[c];
    return s;
}

static int mg_build(mg_t* m, int dim, const int* nel, int n_level, int n_smooth, double omega_boost,
                    const double* K0, const double* w, const uint8_t* con, unsigned w_mask) {
    memset(m, 0, sizeof(*m));
    m->w_mask = w_mask;
    m->dim = dim;
    m->n_level = n_level;
    m->n_smooth = n_smooth;
    m->K0 = K0;
    m->w = w;
    m->con = con;
    m->omega_boost = omega_boost;
    for (int l = 0; l <= n_level; l++) {
        for (int a = 0; a < dim; a++) m->nel[l][a] = nel[a] >> l;
        grid_t g = mkgrid(dim, m->nel[l]);
        m->ndof[l] = g.n_nodes * dim;
        for (int t = 0; t < 5; t++) m->tmp[l][t] = (double*)calloc(m->ndof[l], sizeof(double));
        m->Dinv[l] = (double*)malloc(sizeof(double) * m->ndof[l]);
    }
    /* setup (_solvers.py:442-496) */
    or_diagonal(dim, m->nel[0], K0, w, con, m->Dinv[0]);
    for (long i = 0; i < m->ndof[0]; i++) m->Dinv[0][i] = 1.0 / m->Dinv[0][i];
    const int NB = n_blocks(dim), bs = dim * dim;
    for (int l = 1; l <= n_level; l++) {
        m->A[l] = (double*)malloc(sizeof(double) * (m->ndof[l] / dim) * NB * bs);
        if (l == 1)
            or_galerkin_l0(dim, m->nel[0], K0, w, con, m->A[1]);
        else
            or_galerkin_l1p(dim, m->nel[l - 1], m->A[l - 1], m->A[l]);
        or_stencil_diagonal(dim, m->nel[l], m->A[l], m->Dinv[l]);
        for (long i = 0; i < m->ndof[l]; i++) m->Dinv[l][i] = 1.0 / m->Dinv[l][i];
    }
    long nc = m->ndof[n_level];
    double* dense = (double*)malloc(sizeof(double) * nc * nc);
    m->Lc = (double*)malloc(sizeof(double) * nc * nc);
    or_stencil_to_dense(dim, m->nel[n_level], m->A[n_level], dense);
    int st = or_cholesky((int)nc, dense, 1e-6, m->Lc);
    free(dense);
    return st;
}

static void mg_release(mg_t* m) {
    for (int l = 0; l <= m->n_level; l++) {
        for (int t = 0; t < 5; t++) free(m->tmp[l][t]);
        free(m->Dinv[l]);
        if (l) free(m->A[l]);
    }
    free(m->Lc);
}

/* One V-cycle z = M r from a zero guess with level-0 Jacobi weight omega. */
int or_mg_cycle(int dim, const int* nel, int n_level, int n_smooth, double omega, double omega_boost,
                unsigned w_mask, const double* K0, const double* w, const uint8_t* con, const double* r, double* z);

int or_mg_vcycle(int dim, const int* nel, int n_level, int n_smooth, double omega, double omega_boost,
                 const double* K0, const double* w, const uint8_t* con, const double* r, double* z) {
    return or_mg_cycle(dim, nel, n_level, n_smooth, omega, omega_boost, 0u, K0, w, con, r, z);
}

/* One cycle z = M r from a zero guess; w_mask: levels with the 'w' second correction */
int or_mg_cycle(int dim, const int* nel, int n_level, int n_smooth, double omega, double omega_boost,
                unsigned w_mask, const double* K0, const double* w, const uint8_t* con, const double* r, double* z) {
    mg_t m;
    int st = mg_build(&m, dim, nel, n_level, n_smooth, omega_boost, K0, w, con, w_mask);
    if (st == 0) vcycle(&m, 0, z, r, omega);
    mg_release(&m);
    return st;
}

/* returns iterations; *res = final recursive relative residual; status 0 ok, 1 not
 * converged, 2 coarse factorization failed */
static double wall_s(void) {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

/* Deflation space of the PCG (the library's learned coarse-grid correction, which has no
 * reference counterpart): Q has one column per displacement component c, Q[i][c] = Y[i]
 * where i % dim == c and DOF i is free, else 0; W = A Q, G = Q^T W.  The 3x3 (2x2) G is
 * inverted on the components whose diagonal exceeds 1e-12 of the largest; the others get
 * zero rows and columns.  Deflated PCG of Saad, Yeung, Erhel and Guyomarc'h (SIAM J. Sci.
 * Comput. 21, 2000):  x0 = x + Q G^-1 Q^T (b - A x);  p = z - Q G^-1 W^T z + beta p. */
typedef struct {
    int on, dim;
    long n;
    double *Q, *W; /* dim columns of n */
    double Gi[9];
} defl_t;

static void defl_build(defl_t* d, mg_t* m, const double* Y) {
    memset(d, 0, sizeof(*d));
    if (!Y) return;
    const int dim = m->dim;
    const long n = m->ndof[0];
    d->on = 1;
    d->dim = dim;
    d->n = n;
    d->Q = (double*)calloc((size_t)dim * n, sizeof(double));
    d->W = (double*)calloc((size_t)dim * n, sizeof(double));
    for (long i = 0; i < n; i++)
        if (!(m->con && m->con[i])) d->Q[(i % dim) * n + i] = Y[i];
    for (int c = 0; c < dim; c++) level_matvec(m, 0, d->Q + c * n, d->W + c * n);
    double G[3][3], A[3][3], I[3][3];
    int act[3] = {0, 0, 0};
    double gmax = 0.0;
    for (int c = 0; c < dim; c++)
        for (int e = 0; e < dim; e++) G[c][e] = dot(n, d->Q + c * n, d->W + e * n);
    for (int c = 0; c < dim; c++) gmax = fmax(gmax, G[c][c]);
    for (int c = 0; c < dim; c++) act[c] = gmax > 0.0 && G[c][c] > 1e-12 * gmax;
    for (int c = 0; c < dim; c++)
        for (int e = 0; e < dim; e++) {
            A[c][e] = (act[c] && act[e]) ? 0.5 * (G[c][e] + G[e][c]) : (c == e ? 1.0 : 0.0);
            I[c][e] = c == e ? 1.0 : 0.0;
        }
    for (int k = 0; k < dim; k++) { /* Gauss-Jordan, SPD */
        const double piv = A[k][k];
        for (int j = 0; j < dim; j++) {
            A[k][j] /= piv;
            I[k][j] /= piv;
        }
        for (int i = 0; i < dim; i++)
            if (i != k) {
                const double f = A[i][k];
                for (int j = 0; j < dim; j++) {
                    A[i][j] -= f * A[k][j];
                    I[i][j] -= f * I[k][j];
                }
            }
    }
    for (int c = 0; c < 3; c++)
        for (int e = 0; e < 3; e++) d->Gi[c * 3 + e] = (c < dim && e < dim && act[c] && act[e]) ? I[c][e] : 0.0;
}

/* v -= Q G^-1 (M^T u)  (M = Q or W) when sign < 0, v += ... when sign > 0 */
static void defl_apply(const defl_t* d, const double* M, const double* u, double* v, double sign) {
    const long n = d->n;
    double t[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    for (int k = 0; k < d->dim; k++) t[k] = dot(n, M + k * n, u);
    for (int k = 0; k < d->dim; k++)
        for (int j = 0; j < d->dim; j++) c[k] += d->Gi[k * 3 + j] * t[j];
    for (int k = 0; k < d->dim; k++)
        for (long i = 0; i < n; i++) v[i] += sign * c[k] * d->Q[k * n + i];
}

static void defl_free(defl_t* d) {
    free(d->Q);
    free(d->W);
}

static int mgcg_core(int dim, const int* nel, int n_level, int n_smooth, double omega, double min_omega_arg,
                     double omega_boost, double tol, int maxiter, const double* K0, const double* w,
                     const uint8_t* con, const double* rhs, double* x, int use_x0, double* res_out,
                     int* status_out, double* times_out, const double* Y, unsigned w_mask, double fixed_omega) {
    mg_t m;
    const double t0 = wall_s();
    int st = mg_build(&m, dim, nel, n_level, n_smooth, omega_boost, K0, w, con, w_mask);
    const double t1 = wall_s();
    int iters = 0;
    double R = 0.0;
    int status = 0;
    if (st != 0) {
        status = 2;
    } else {
        long n = m.ndof[0];
        double max_omega = omega, min_omega = fmax(omega / 2.0, min_omega_arg), d_omega = max_omega - min_omega;
        if (fixed_omega > 0.0) { /* a fixed weight: the schedule's floor with no span */
            min_omega = fixed_omega;
            d_omega = 0.0;
        }
        double cur = min_omega;
        double *r = (double*)malloc(sizeof(double) * n), *z = (double*)malloc(sizeof(double) * n);
        double *p = (double*)malloc(sizeof(double) * n), *q = (double*)malloc(sizeof(double) * n);
        if (!use_x0) memset(x, 0, sizeof(double) * n);
        defl_t D;
        defl_build(&D, &m, Y);
        level_matvec(&m, 0, x, q);
        for (long i = 0; i < n; i++) r[i] = rhs[i] - q[i];
        if (D.on) {
            defl_apply(&D, D.Q, r, x, 1.0);
            level_matvec(&m, 0, x, q);
            for (long i = 0; i < n; i++) r[i] = rhs[i] - q[i];
        }
        vcycle(&m, 0, z, r, cur);
        memcpy(p, z, sizeof(double) * n);
        if (D.on) defl_apply(&D, D.W, z, p, -1.0);
        double rho_old = dot(n, r, z);
        double norm_b = sqrt(dot(n, rhs, rhs));
        status = 1;
        for (int it = 0; it < maxiter; it++) {
            level_matvec(&m, 0, p, q);
            double alpha = rho_old / dot(n, p, q);
#pragma omp parallel for
            for (long i = 0; i < n; i++) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            R = sqrt(dot(n, r, r)) / norm_b;
            iters = it + 1;
            if (R < tol) {
                status = 0;
                break;
            }
            double cl = R < tol ? tol : (R > 0.1 ? 0.1 : R);
            cur = min_omega + d_omega / 2.0 * exp((-cl + tol) * 500.0);
            vcycle(&m, 0, z, r, cur);
            double rho_new = dot(n, r, z);
            double beta = rho_new / rho_old;
#pragma omp parallel for
            for (long i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
            if (D.on) defl_apply(&D, D.W, z, p, -1.0);
            rho_old = rho_new;
        }
        free(r); free(z); free(p); free(q);
        defl_free(&D);
    }
    if (times_out) {
        times_out[0] = t1 - t0;
        times_out[1] = wall_s() - t1;
    }
    mg_release(&m);
    *res_out = R;
    *status_out = status;
    return iters;
}

/* or_mgcg_solve with wall-clock seconds of the hierarchy setup (times_out[0]) and of the
 * PCG start plus iterations (times_out[1]); times_out may be NULL */
int or_mgcg_solve_timed(int dim, const int* nel, int n_level, int n_smooth, double omega, double min_omega_arg,
                        double omega_boost, double tol, int maxiter, const double* K0, const double* w,
                        const uint8_t* con, const double* rhs, double* x, int use_x0, double* res_out,
                        int* status_out, double* times_out) {
    return mgcg_core(dim, nel, n_level, n_smooth, omega, min_omega_arg, omega_boost, tol, maxiter, K0, w, con, rhs, x,
                     use_x0, res_out, status_out, times_out, NULL, 0u, 0.0);
}

/* or_mgcg_solve with the deflation space spanned by the components of the nodal field Y */
int or_mgcg_solve_deflated(int dim, const int* nel, int n_level, int n_smooth, double omega, double min_omega_arg,
                           double omega_boost, double tol, int maxiter, const double* K0, const double* w,
                           const uint8_t* con, const double* rhs, double* x, int use_x0, const double* Y,
                           double* res_out, int* status_out) {
    return mgcg_core(dim, nel, n_level, n_smooth, omega, min_omega_arg, omega_boost, tol, maxiter, K0, w, con, rhs, x,
                     use_x0, res_out, status_out, NULL, Y, 0u, 0.0);
}

/* or_mgcg_solve with the 'w' cycle's second coarse correction at the levels of w_mask */
int or_mgcg_solve_w(int dim, const int* nel, int n_level, int n_smooth, double omega, double min_omega_arg,
                    double omega_boost, double tol, int maxiter, const double* K0, const double* w,
                    const uint8_t* con, const double* rhs, double* x, int use_x0, unsigned w_mask, double* res_out,
                    int* status_out) {
    return mgcg_core(dim, nel, n_level, n_smooth, omega, min_omega_arg, omega_boost, tol, maxiter, K0, w, con, rhs, x,
                     use_x0, res_out, status_out, NULL, NULL, w_mask, 0.0);
}

/* The general form: deflation field Y (may be NULL), 'w' cycle levels w_mask and a fixed
 * Jacobi weight (fixed_omega > 0; 0 = the reference's schedule) */
int or_mgcg_solve_ex(int dim, const int* nel, int n_level, int n_smooth, double omega, double min_omega_arg,
                     double omega_boost, double tol, int maxiter, const double* K0, const double* w,
                     const uint8_t* con, const double* rhs, double* x, int use_x0, const double* Y, unsigned w_mask,
                     double fixed_omega, double* res_out, int* status_out) {
    return mgcg_core(dim, nel, n_level, n_smooth, omega, min_omega_arg, omega_boost, tol, maxiter, K0, w, con, rhs, x,
                     use_x0, res_out, status_out, NULL, Y, w_mask, fixed_omega);
}

int or_mgcg_solve(int dim, const int* nel, int n_level, int n_smooth, double omega, double min_omega_arg,
                  double omega_boost, double tol, int maxiter, const double* K0, const double* w,
                  const uint8_t* con, const double* rhs, double* x, int use_x0, double* res_out,
                  int* status_out) {
    return or_mgcg_solve_timed(dim, nel, n_level, n_smooth, omega, min_omega_arg, omega_boost, tol, maxiter, K0, w,
                               con, rhs, x, use_x0, res_out, status_out, NULL);
}

/* ------------------------------------------------------------------------------------
 * Unpreconditioned CG on the structured operator: the reference CG solver
 * (solvers/CUDA/_solvers.py:114-127) calls cupyx.scipy.sparse.linalg.cg(kernel, rhs,
 * x0, tol, maxiter), which is textbook CG with the identity preconditioner:
 *   r = b - A x; rho = r.r; p = r (first iteration) or r + (rho / rho_prev) p;
 *   q = A p; alpha = rho / p.q; x += alpha p; r -= alpha q;
 *   stop when ||r|| <= tol ||b|| (atol = max(0, tol ||b||)) or after maxiter iterations;
 *   b = 0 returns x = 0.
 * Returns the iterations; *res_out = ||r|| / ||b|| (recursive residual).
 * ---------------------------------------------------------------------------------- */
int or_cg_solve(int dim, const int* nel, const double* K0, const double* w, const uint8_t* con, const double* rhs,
                double* x, int use_x0, double tol, int maxiter, double* res_out) {
    grid_t g = mkgrid(dim, nel);
    const long n = g.n_nodes * dim;
    double *r = (double*)malloc(sizeof(double) * n), *p = (double*)malloc(sizeof(double) * n);
    double* q = (double*)malloc(sizeof(double) * n);
    const double nb = sqrt(dot(n, rhs, rhs));
    int iters = 0;
    double R = 0.0;
    if (nb == 0.0) {
        memset(x, 0, sizeof(double) * n);
    } else {
        if (!use_x0) memset(x, 0, sizeof(double) * n);
        or_matvec(dim, nel, K0, w, x, con, q);
        for (long i = 0; i < n; i++) r[i] = rhs[i] - q[i];
        const double atol = tol * nb;
        double rho = 0.0, rho_prev = 0.0;
        for (int it = 0; it < maxiter; it++) {
            rho_prev = rho;
            rho = dot(n, r, r);
            if (it == 0) {
                memcpy(p, r, sizeof(double) * n);
            } else {
                const double beta = rho / rho_prev;
#pragma omp parallel for
                for (long i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
            }
            or_matvec(dim, nel, K0, w, p, con, q);
            const double alpha = rho / dot(n, p, q);
#pragma omp parallel for
            for (long i = 0; i < n; i++) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            iters = it + 1;
            const double rn = sqrt(dot(n, r, r));
            R = rn / nb;
            if (rn <= atol) break;
        }
    }
    free(r); free(p); free(q);
    *res_out = R;
    return iters;
}

/* ------------------------------------------------------------------------------------
 * Cone density filter (filters.cu:1-154, core/CPU/_filter.py:7-125).
 * offsets: K x dim ints, weights: K doubles (already normalised to sum 1).
 * ---------------------------------------------------------------------------------- */
static inline long el_lin(int dim, const int* nel, int i, int j, int k) {
    return dim == 3 ? (long)i * nel[1] * nel[2] + (long)j * nel[2] + k : (long)i * nel[1] + j;
}
static inline int el_in(int dim, const int* nel, int i, int j, int k) {
    if (i < 0 || j < 0 || i >= nel[0] || j >= nel[1]) return 0;
    return dim == 3 ? (k >= 0 && k < nel[2]) : 1;
}
static inline void el_ijk(int dim, const int* nel, long e, int* i, int* j, int* k) {
    if (dim == 3) {
        *i = (int)(e / ((long)nel[1] * nel[2]));
        *j = (int)((e / nel[2]) % nel[1]);
        *k = (int)(e % nel[2]);
    } else {
        *i = (int)(e / nel[1]);
        *j = (int)(e % nel[1]);
        *k = 0;
    }
}

void or_filter_normalizer(int dim, const int* nel, int K, const int* offsets, const double* weights, double* norm) {
    long ne = dim == 3 ? (long)nel[0] * nel[1] * nel[2] : (long)nel[0] * nel[1];
#pragma omp parallel for
    for (long e = 0; e < ne; e++) {
        int i, j, k;
        el_ijk(dim, nel, e, &i, &j, &k);
        double s = 0.0;
        for (int q = 0; q < K; q++) {
            int a = i + offsets[q * dim], b = j + offsets[q * dim + 1], c = dim == 3 ? k + offsets[q * dim + 2] : 0;
            if (el_in(dim, nel, a, b, c)) s += weights[q];
        }
        norm[e] = s;
    }
}

void or_filter_fwd(int dim, const int* nel, int K, const int* offsets, const double* weights, const double* v,
                   double* out) {
    long ne = dim == 3 ? (long)nel[0] * nel[1] * nel[2] : (long)nel[0] * nel[1];
#pragma omp parallel for
    for (long e = 0; e < ne; e++) {
        int i, j, k;
        el_ijk(dim, nel, e, &i, &j, &k);
        double sv = 0.0, sw = 0.0;
        for (int q = 0; q < K; q++) {
            int a = i + offsets[q * dim], b = j + offsets[q * dim + 1], c = dim == 3 ? k + offsets[q * dim + 2] : 0;
            if (!el_in(dim, nel, a, b, c)) continue;
            sv += weights[q] * v[el_lin(dim, nel, a, b, c)];
            sw += weights[q];
        }
        out[e] = sw > 0 ? sv / sw : 0.0;
    }
}

void or_filter_adj(int dim, const int* nel, int K, const int* offsets, const double* weights, const double* norm,
                   const double* v, double* out) {
    long ne = dim == 3 ? (long)nel[0] * nel[1] * nel[2] : (long)nel[0] * nel[1];
#pragma omp parallel for
    for (long e = 0; e < ne; e++) {
        int i, j, k;
        el_ijk(dim, nel, e, &i, &j, &k);
        double s = 0.0;
        for (int q = 0; q < K; q++) {
            int a = i + offsets[q * dim], b = j + offsets[q * dim + 1], c = dim == 3 ? k + offsets[q * dim + 2] : 0;
            if (!el_in(dim, nel, a, b, c)) continue;
            long jd = el_lin(dim, nel, a, b, c);
            s += (weights[q] / norm[jd]) * v[jd];
        }
        out[e] = s;
    }
}

/* ------------------------------------------------------------------------------------
 * OC update (Optimizers/CUDA/OC.py:67-129, single constraint):
 *   ocP = x * sqrt(max(-df/dg, 0)) (NaN -> 0; all-zero -> 1e-3),
 *   bisection on l in [1e-9, 1e9] until (l2-l1)/(l2+l1) <= 1e-8, testing
 *   g(x_new) = dg . x_new - vf <= 0 with x_new = max(0, max(xL, min(1, min(xU, ocP/l)))).
 * dg is a per-element vector (A_e / V).  Returns the number of bisection steps.
 * ---------------------------------------------------------------------------------- */
int or_oc_update(long n, const double* x, const double* df, const double* dg, double vf, double move,
                 double* x_new) {
    double* ocp = (double*)malloc(sizeof(double) * n);
    double abs_sum = 0.0;
    for (long i = 0; i < n; i++) {
        double t = -df[i] / dg[i];
        t = t > 0 ? t : 0.0;
        double s = sqrt(t);
        if (isnan(s)) s = 0.0;
        ocp[i] = x[i] * s;
        abs_sum += fabs(ocp[i]);
    }
    if (abs_sum == 0.0)
        for (long i = 0; i < n; i++) ocp[i] = 1e-3;
    double l1 = 1e-9, l2 = 1e9;
    int steps = 0;
    while ((l2 - l1) / (l2 + l1) > 1e-8) {
        double lmid = (l1 + l2) / 2.0;
        double g = 0.0;
        for (long i = 0; i < n; i++) {
            double xu = fmin(fmax(x[i] + move, 0.0), 1.0), xl = fmin(fmax(x[i] - move, 0.0), 1.0);
            double v = fmax(0.0, fmax(xl, fmin(1.0, fmin(xu, ocp[i] / lmid))));
            x_new[i] = v;
            g += dg[i] * v;
        }
        g -= vf;
        if (g <= 0.0)
            l2 = lmid;
        else
            l1 = lmid;
        steps++;
    }
    free(ocp);
    return steps;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
