// Explicit CSR assembly of the structured stiffness matrix: the reference's
// StructuredStiffnessKernel.construct (pyFANTOM/stiffness/CUDA/_FEA.py:484-516, which forms
// K I with its node-basis matmat kernels), built here directly from the element matrix.
//
// The matrix is the one the library's matvec applies: Z K Z + (I - Z), with Z zeroing the
// constrained DOFs (rows and columns of a constrained DOF are those of the identity).  Row
// (node n, component a) holds, for every node m within one element of n (in increasing
// node index) and every component b, sum over the elements e containing n and m of
// E_e K0[(l_n(e), a), (l_m(e), b)].  Entries are kept even where they are zero (constrained
// couplings), so the sparsity pattern depends on the grid only: a node has
// c(i) c(j) c(k) neighbours with c = 2 on a boundary plane and 3 inside, and the row
// pointers follow in closed form.  One thread per row, no atomics.
#include "common.cuh"
#include "elemop.cuh"

namespace pf {

// neighbours along one axis of a node at index v of nn nodes, and their prefix over v' < v
__host__ __device__ __forceinline__ long long nb1(int v, int nn) { return 1 + (v > 0) + (v < nn - 1); }
__host__ __device__ __forceinline__ long long nbp(int v) { return v == 0 ? 0 : 2 + 3LL * (v - 1); }

// local corner of an element from its offsets (bx, by, bz) in {0, 1} (reference order)
__device__ __forceinline__ int corner_of(int bx, int by, int bz) { return bz * 4 + (by ? (bx ? 2 : 3) : (bx ? 1 : 0)); }

template <int DIM>
__global__ void __launch_bounds__(256) k_construct_csr(Grid g, const double* __restrict__ E,
                                                       const uint8_t* __restrict__ mask,
                                                       const double* __restrict__ K0, int* __restrict__ row_ptr,
                                                       int* __restrict__ col, double* __restrict__ val) {
    constexpr int DOF = DIM;
    constexpr int ND = DIM == 3 ? 24 : 8;  // element matrix order
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.n_nodes * DOF) return;
    const long long n = t / DOF;
    const int a = (int)(t % DOF);
    const int nx = g.nn[0], ny = g.nn[1], nz = DIM == 3 ? g.nn[2] : 1;
    int i, j, k;
    if (DIM == 3) {
        k = (int)(n % nz);
        i = (int)((n / nz) % nx);
        j = (int)(n / ((long long)nz * nx));
    } else {
        i = (int)(n % nx);
        j = (int)(n / nx);
        k = 0;
    }
    const long long sx = 3LL * nx - 2, sz = DIM == 3 ? 3LL * nz - 2 : 1;
    const long long cx = nb1(i, nx), cy = nb1(j, ny), cz = DIM == 3 ? nb1(k, nz) : 1;
    const long long before =
        DIM == 3 ? nbp(j) * sx * sz + cy * nbp(i) * sz + cy * cx * nbp(k) : nbp(j) * sx + cy * nbp(i);
    const long long cnt = cx * cy * cz;
    long long p = (long long)DOF * DOF * before + (long long)a * cnt * DOF;
    row_ptr[t] = (int)p;
    if (t == g.n_nodes * DOF - 1) row_ptr[t + 1] = (int)(p + cnt * DOF);
    const uint8_t mn = mask ? mask[n] : (uint8_t)0;
    const bool row_con = (mn >> a) & 1;
    const int kr = DIM == 3 ? 1 : 0;
    for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++)
            for (int dz = -kr; dz <= kr; dz++) {
                const int mi = i + dx, mj = j + dy, mk = k + dz;
                if (mi < 0 || mj < 0 || mk < 0 || mi >= nx || mj >= ny || mk >= nz) continue;
                const long long m = DIM == 3 ? (long long)mk + (long long)nz * (mi + (long long)nx * mj)
                                             : (long long)mi + (long long)nx * mj;
                const uint8_t mm = mask ? mask[m] : (uint8_t)0;
                double v[DOF];
#pragma unroll
                for (int b = 0; b < DOF; b++) v[b] = 0.0;
                if (row_con) {
                    if (m == n) v[a] = 1.0;
                } else {
                    // elements containing n and m: lower corner within [max-1, min] per axis
                    const int x0 = max(max(i, mi) - 1, 0), x1 = min(min(i, mi), g.nel[0] - 1);
                    const int y0 = max(max(j, mj) - 1, 0), y1 = min(min(j, mj), g.nel[1] - 1);
                    const int z0 = DIM == 3 ? max(max(k, mk) - 1, 0) : 0;
                    const int z1 = DIM == 3 ? min(min(k, mk), g.nel[2] - 1) : 0;
                    for (int ex = x0; ex <= x1; ex++)
                        for (int ey = y0; ey <= y1; ey++)
                            for (int ez = z0; ez <= z1; ez++) {
                                const long long e = DIM == 3 ? ((long long)ex * g.nel[1] + ey) * g.nel[2] + ez
                                                             : (long long)ex * g.nel[1] + ey;
                                const double w = E[e];
                                const int ln = corner_of(i - ex, j - ey, k - ez), lm = corner_of(mi - ex, mj - ey, mk - ez);
#pragma unroll
                                for (int b = 0; b < DOF; b++) v[b] += w * K0[(ln * DOF + a) * ND + lm * DOF + b];
                            }
#pragma unroll
                    for (int b = 0; b < DOF; b++)
                        if ((mm >> b) & 1) v[b] = 0.0;
                }
#pragma unroll
                for (int b = 0; b < DOF; b++) {
                    col[p] = (int)(m * DOF + b);
                    val[p] = v[b];
                    p++;
                }
            }
}

long long csr_nnz(const Grid& g) {
    const long long sx = 3LL * g.nn[0] - 2, sy = 3LL * g.nn[1] - 2, sz = g.dim == 3 ? 3LL * g.nn[2] - 2 : 1;
    return (long long)g.dof * g.dof * sx * sy * sz;
}

int launch_construct_csr(const Grid& g, const double* E, const uint8_t* mask, const double* K0_dev, int* row_ptr,
                         int* col, double* val, cudaStream_t st) {
    if (csr_nnz(g) >= (1LL << 31) || g.n_nodes * g.dof >= (1LL << 31))
        return fail(PF_UNSUPPORTED, "construct: %lld nonzeros exceed 32-bit indices", csr_nnz(g));
    const long long rows = g.n_nodes * g.dof;
    const unsigned nb = (unsigned)((rows + 255) / 256);
    pf::count_launch();
    if (g.dim == 3)
        k_construct_csr<3><<<nb, 256, 0, st>>>(g, E, mask, K0_dev, row_ptr, col, val);
    else
        k_construct_csr<2><<<nb, 256, 0, st>>>(g, E, mask, K0_dev, row_ptr, col, val);
    PF_LAUNCH_CHECK("construct launch");
    return PF_OK;
}

}  // namespace pf
