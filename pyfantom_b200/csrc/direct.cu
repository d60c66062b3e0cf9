// Direct solve of K(E) u = b for small structured problems: the drop-in for the reference's
// SPSOLVE (pyFANTOM/solvers/CUDA/_solvers.py:245-328), which assembles K in CSR
// (StructuredStiffnessKernel.construct, stiffness/CUDA/_FEA.py:484-516), keeps the free
// rows and columns and calls a sparse direct solver; constrained entries of the solution
// are the right-hand side's.
//
// Here the free-DOF matrix is assembled dense (one thread per free row gathers its entries
// from the row node's adjacent elements, so every entry is written by one thread in a fixed
// order), factored by the tiled Cholesky of the coarse solver (L L^T, inverse factor
// L^-1), and the solution is x = L^-T (L^-1 b) by two dense matvecs.  Meant for problems
// up to kDirectMaxFree free DOFs (the matrix and its inverse factor held dense).
#include <vector>

#include "common.cuh"
#include "elemop.cuh"
#include "mgkern.cuh"

constexpr int kDirectMaxFree = 20480;

struct pf_direct {
    const pf::Op* op = nullptr;
    pf::Dense dense;
    double* K0 = nullptr;  // device copy of the element matrix
    double* bf = nullptr;  // free right-hand side / intermediate
    double* xf = nullptr;
    int n = 0;
};

namespace pf {

// row thread: free DOF r = global DOF g; M[r][f(gc)] += E_e K0[a*dof + comp][b*dof + c]
template <int DIM>
__global__ void k_direct_assemble(Grid g, const double* __restrict__ E, const double* __restrict__ K0,
                                  const int* __restrict__ free_dofs, const int* __restrict__ dof_to_free, int n,
                                  int np, double* __restrict__ M) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    constexpr int NC = DIM == 3 ? 8 : 4, ND = NC * DIM;
    const int gdof = free_dofs[r];
    const int node = gdof / DIM, comp = gdof - node * DIM;
    int i, j, k = 0;
    if (DIM == 3) {
        const int t = node / g.nn[2];
        k = node - t * g.nn[2];
        j = t / g.nn[0];
        i = t - j * g.nn[0];
    } else {
        j = node / g.nn[0];
        i = node - j * g.nn[0];
    }
    double* row = M + (long long)r * np;
    for (int a = 0; a < NC; a++) {  // the row node is corner a of element (i, j, k) - corner(a)
        const int ei = i - kCXd(a), ej = j - kCYd(a), ek = DIM == 3 ? k - kCZd(a) : 0;
        if (ei < 0 || ej < 0 || ei >= g.nel[0] || ej >= g.nel[1]) continue;
        if (DIM == 3 && (ek < 0 || ek >= g.nel[2])) continue;
        const long long e = DIM == 3 ? ((long long)ei * g.nel[1] + ej) * g.nel[2] + ek : (long long)ei * g.nel[1] + ej;
        const double w = E[e];
        const double* Kr = K0 + (a * DIM + comp) * ND;
        for (int b = 0; b < NC; b++) {
            const int bi = ei + kCXd(b), bj = ej + kCYd(b), bk = DIM == 3 ? ek + kCZd(b) : 0;
            const long long bn = DIM == 3 ? (long long)bk + (long long)g.nn[2] * (bi + (long long)g.nn[0] * bj)
                                           : (long long)bi + (long long)g.nn[0] * bj;
            for (int c = 0; c < DIM; c++) {
                const int fc = dof_to_free[bn * DIM + c];
                if (fc >= 0) row[fc] += w * Kr[b * DIM + c];
            }
        }
    }
}

__global__ void k_gather(int n, const int* __restrict__ idx, const double* __restrict__ src, double* __restrict__ dst) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) dst[r] = src[idx[r]];
}
__global__ void k_scatter(int n, const int* __restrict__ idx, const double* __restrict__ src, double* __restrict__ dst) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) dst[idx[r]] = src[r];
}

// y = L^-1 b: warp per row, lower triangle only
__global__ void __launch_bounds__(256) k_lower_matvec(const double* __restrict__ Li, int np, int n,
                                                      const double* __restrict__ b, double* __restrict__ y) {
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5), l = threadIdx.x & 31;
    if (row >= n) return;
    const double* Lr = Li + (long long)row * np;
    double s = 0.0;
    for (int c = l; c <= row; c += 32) s += Lr[c] * b[c];
    s = warp_sum(s);
    if (l == 0) y[row] = s;
}

// x = L^-T y: warp per group of 32 columns, coalesced rows i >= column
__global__ void __launch_bounds__(256) k_lower_tmatvec(const double* __restrict__ Li, int np, int n,
                                                       const double* __restrict__ y, double* __restrict__ x) {
    const int grp = blockIdx.x * 8 + (threadIdx.x >> 5), l = threadIdx.x & 31;
    const int col = grp * 32 + l;
    if (grp * 32 >= n) return;
    double s = 0.0;
    for (int i = grp * 32; i < n; i++)
        if (col < n && i >= col) s += Li[(long long)i * np + col] * y[i];
    if (col < n) x[col] = s;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_direct_create(const pf_op* op, pf_direct** out) {
    if (!op || !out) return fail(PF_BAD_ARG, "pf_direct_create: NULL argument");
    auto* d = new pf_direct();
    d->op = op;
    const int nd = (op->grid.dim == 3 ? 8 : 4) * op->grid.dim;
    if (cudaMalloc(&d->K0, sizeof(double) * nd * nd) != cudaSuccess) {
        delete d;
        return fail(PF_NO_MEMORY, "pf_direct_create: allocation failed");
    }
    if (cudaMemcpy(d->K0, op->K0, sizeof(double) * nd * nd, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d->K0);
        delete d;
        return fail(PF_CUDA_ERROR, "pf_direct_create: copy of K0 failed");
    }
    *out = d;
    return PF_OK;
}

extern "C" int pf_direct_destroy(pf_direct* d) {
    if (!d) return PF_OK;
    dense_free(&d->dense);
    for (void* p : {(void*)d->K0, (void*)d->bf, (void*)d->xf})
        if (p) cudaFree(p);
    delete d;
    return PF_OK;
}

static int direct_reserve(pf_direct* d, int n) {
    if (d->n == n && d->dense.M) return PF_OK;
    dense_free(&d->dense);
    if (d->bf) cudaFree(d->bf);
    if (d->xf) cudaFree(d->xf);
    d->bf = d->xf = nullptr;
    d->n = 0;
    int s = dense_alloc(&d->dense, n);
    if (s) return s;
    if (cudaMalloc(&d->bf, sizeof(double) * n) != cudaSuccess || cudaMalloc(&d->xf, sizeof(double) * n) != cudaSuccess)
        return fail(PF_NO_MEMORY, "pf_direct_solve_f64: allocation failed");
    d->n = n;
    return PF_OK;
}

extern "C" int pf_direct_solve_f64(pf_direct* d, const double* E, const int* free_dofs, const int* dof_to_free,
                                   int n_free, const double* b, double* x, void* stream) {
    if (!d || !E || !free_dofs || !dof_to_free || !b || !x || n_free < 1)
        return fail(PF_BAD_ARG, "pf_direct_solve_f64: bad argument");
    if (n_free > kDirectMaxFree)
        return fail(PF_BAD_ARG, "pf_direct_solve_f64: %d free DOFs exceed the dense direct solver's limit of %d",
                    n_free, kDirectMaxFree);
    int s = direct_reserve(d, n_free);
    if (s) return s;
    cudaStream_t st = as_stream(stream);
    Dense& D = d->dense;
    const Grid& g = d->op->grid;
    const long long ndof = g.n_nodes * g.dof;
    PF_CUDA(cudaMemsetAsync(D.M, 0, (size_t)D.np * D.np * sizeof(double), st));
    count_launch();
    if (g.dim == 3)
        k_direct_assemble<3><<<(n_free + 127) / 128, 128, 0, st>>>(g, E, d->K0, free_dofs, dof_to_free, n_free, D.np,
                                                                   D.M);
    else
        k_direct_assemble<2><<<(n_free + 127) / 128, 128, 0, st>>>(g, E, d->K0, free_dofs, dof_to_free, n_free, D.np,
                                                                   D.M);
    PF_LAUNCH_CHECK("direct assembly launch");
    if ((s = dense_factor_linv(&D, 0.0, st))) return s;
    // x = b (constrained entries keep the right-hand side), then the free entries
    PF_CUDA(cudaMemcpyAsync(x, b, sizeof(double) * ndof, cudaMemcpyDeviceToDevice, st));
    count_launch(4);
    k_gather<<<(n_free + 255) / 256, 256, 0, st>>>(n_free, free_dofs, b, d->bf);
    k_lower_matvec<<<(n_free + 7) / 8, 256, 0, st>>>(D.Linv, D.np, n_free, d->bf, d->xf);
    k_lower_tmatvec<<<((n_free + 31) / 32 + 7) / 8, 256, 0, st>>>(D.Linv, D.np, n_free, d->xf, d->bf);
    k_scatter<<<(n_free + 255) / 256, 256, 0, st>>>(n_free, free_dofs, d->bf, x);
    PF_LAUNCH_CHECK("direct solve launch");
    int fpiv = 0;
    PF_CUDA(cudaMemcpyAsync(&fpiv, D.fail, sizeof(int), cudaMemcpyDeviceToHost, st));
    PF_CUDA(cudaStreamSynchronize(st));
    if (fpiv) return fail(PF_FACTOR_FAILED, "pf_direct_solve_f64: matrix not positive definite (pivot %d)", fpiv - 1);
    return PF_OK;
}
