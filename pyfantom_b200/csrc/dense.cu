// Dense FP64 coarse solver on the device.
//
// The reference factors the coarsest Galerkin operator with CHOLMOD on the host as
// A_L + beta I, beta = 1e-6 (pyFANTOM/solvers/CUDA/_solvers.py:508-514), and copies every
// coarse right-hand side to the host and back.  Here the factorisation stays on the GPU:
// a right-looking blocked Cholesky with 32x32 tiles (diagonal tile in shared memory,
// triangular solve of the panel, symmetric rank-32 update of the trailing matrix),
// followed by the inverse of the factor and the explicit inverse A^-1 = L^-T L^-1.  A
// coarse solve is then one dense matrix-vector product, spread over many warps, with no
// host round trip.
#include "common.cuh"
#include "mgkern.cuh"

namespace pf {

constexpr int TB = 32;

__global__ void k_pad_diag(double* M, int n, int np, double beta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < np) M[(long long)i * np + i] += i < n ? beta : 1.0;
}

__global__ void __launch_bounds__(1024) k_potrf_tile(double* M, int np, int p, int* fail) {
    __shared__ double s[TB][TB + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    double* T = M + (long long)(p * TB) * np + p * TB;
    s[ty][tx] = T[(long long)ty * np + tx];
    __syncthreads();
    for (int j = 0; j < TB; j++) {
        if (tx == j && ty == j) {
            double v = s[j][j];
            if (!(v > 0.0)) {
                atomicCAS(fail, 0, p * TB + j + 1);
                v = 1.0;
            }
            s[j][j] = sqrt(v);
        }
        __syncthreads();
        if (tx == j && ty > j) s[ty][j] /= s[j][j];
        __syncthreads();
        if (ty > j && tx > j && tx <= ty) s[ty][tx] -= s[ty][j] * s[tx][j];
        __syncthreads();
    }
    T[(long long)ty * np + tx] = tx <= ty ? s[ty][tx] : 0.0;
}

// tile(i,p) <- tile(i,p) * L_pp^{-T}, i = p+1+blockIdx.x ; one thread per tile row
__global__ void __launch_bounds__(TB) k_trsm(double* M, int np, int p) {
    __shared__ double L[TB][TB + 1];
    const int r = threadIdx.x;
    const double* Lpp = M + (long long)(p * TB) * np + p * TB;
    for (int q = 0; q < TB; q++) L[q][r] = Lpp[(long long)q * np + r];
    __syncthreads();
    const int i = p + 1 + blockIdx.x;
    double* row = M + (long long)(i * TB + r) * np + p * TB;
    double x[TB];
#pragma unroll
    for (int j = 0; j < TB; j++) {
        double s = row[j];
#pragma unroll
        for (int k = 0; k < j; k++) s -= x[k] * L[j][k];
        x[j] = s / L[j][j];
    }
#pragma unroll
    for (int j = 0; j < TB; j++) row[j] = x[j];
}

// trailing update: tile(i,k) -= L_ip L_kp^T for p < k <= i
__global__ void __launch_bounds__(1024) k_syrk(double* M, int np, int p) {
    __shared__ double A[TB][TB + 1], B[TB][TB + 1];
    // decode lower-triangular pair index -> (i, k) relative to p+1
    const int t = blockIdx.x;
    int ii = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((ii + 1) * (ii + 2) / 2 <= t) ii++;
    while (ii * (ii + 1) / 2 > t) ii--;
    const int kk = t - ii * (ii + 1) / 2;
    const int i = p + 1 + ii, k = p + 1 + kk;
    const int tx = threadIdx.x, ty = threadIdx.y;
    A[ty][tx] = M[(long long)(i * TB + ty) * np + p * TB + tx];
    B[ty][tx] = M[(long long)(k * TB + ty) * np + p * TB + tx];
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < TB; q++) s += A[ty][q] * B[tx][q];
    M[(long long)(i * TB + ty) * np + k * TB + tx] -= s;
}

// Linv diagonal tiles: inverse of each lower-triangular L_pp (thread c -> column c)
__global__ void __launch_bounds__(TB) k_trtri_tiles(const double* M, double* Linv, int np) {
    __shared__ double L[TB][TB + 1];
    const int p = blockIdx.x, c = threadIdx.x;
    const double* Lpp = M + (long long)(p * TB) * np + p * TB;
    for (int q = 0; q < TB; q++) L[q][c] = Lpp[(long long)q * np + c];
    __syncthreads();
    double x[TB];
#pragma unroll
    for (int r = 0; r < TB; r++) {
        double s = (r == c) ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < r; k++) s -= L[r][k] * x[k];
        x[r] = r < c ? 0.0 : s / L[r][r];
    }
    double* out = Linv + (long long)(p * TB) * np + p * TB;
#pragma unroll
    for (int r = 0; r < TB; r++) out[(long long)r * np + c] = x[r];
}

// Linv_ip = -Linv_ii * sum_{k=p}^{i-1} L_ik Linv_kp   (p = blockIdx.x < i)
__global__ void __launch_bounds__(1024) k_linv_row(const double* M, double* Linv, int np, int i) {
    __shared__ double A[TB][TB + 1], B[TB][TB + 1];
    const int p = blockIdx.x, tx = threadIdx.x, ty = threadIdx.y;
    double s = 0.0;
    for (int k = p; k < i; k++) {
        A[ty][tx] = M[(long long)(i * TB + ty) * np + k * TB + tx];
        B[ty][tx] = Linv[(long long)(k * TB + ty) * np + p * TB + tx];
        __syncthreads();
#pragma unroll
        for (int q = 0; q < TB; q++) s += A[ty][q] * B[q][tx];
        __syncthreads();
    }
    B[ty][tx] = s;
    A[ty][tx] = Linv[(long long)(i * TB + ty) * np + i * TB + tx];
    __syncthreads();
    double o = 0.0;
#pragma unroll
    for (int q = 0; q < TB; q++) o += A[ty][q] * B[q][tx];
    Linv[(long long)(i * TB + ty) * np + p * TB + tx] = -o;
}

// Ainv(a,b) = sum_{k >= max(a,b)} Linv_ka^T Linv_kb
__global__ void __launch_bounds__(1024) k_ainv(const double* Linv, double* Ainv, int np, int nt) {
    __shared__ double A[TB][TB + 1], B[TB][TB + 1];
    const int a = blockIdx.x, b = blockIdx.y, tx = threadIdx.x, ty = threadIdx.y;
    const int k0 = a > b ? a : b;
    double s = 0.0;
    for (int k = k0; k < nt; k++) {
        A[ty][tx] = Linv[(long long)(k * TB + ty) * np + a * TB + tx];
        B[ty][tx] = Linv[(long long)(k * TB + ty) * np + b * TB + tx];
        __syncthreads();
#pragma unroll
        for (int q = 0; q < TB; q++) s += A[q][ty] * B[q][tx];
        __syncthreads();
    }
    Ainv[(long long)(a * TB + ty) * np + b * TB + tx] = s;
}

// x = Ainv b (rows < n), one warp per row, accumulation in FP64
template <typename T>
__global__ void __launch_bounds__(256) k_dense_matvec(const double* __restrict__ Ainv, int np, int n,
                                                      const T* __restrict__ b, T* __restrict__ x, const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (skip && *skip) return;
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5), l = threadIdx.x & 31;
    if (row >= n) return;
    const double* Ar = Ainv + (long long)row * np;
    double s = 0.0;
    for (int c = l; c < n; c += 32) s += Ar[c] * (double)b[c];
    s = warp_sum(s);
    if (l == 0) x[row] = (T)s;
}

int dense_alloc(Dense* d, int n) {
    d->n = n;
    d->np = (n + TB - 1) / TB * TB;
    const size_t bytes = (size_t)d->np * d->np * sizeof(double);
    if (cudaMalloc(&d->M, bytes) != cudaSuccess || cudaMalloc(&d->Linv, bytes) != cudaSuccess ||
        cudaMalloc(&d->Ainv, bytes) != cudaSuccess || cudaMalloc(&d->fail, sizeof(int)) != cudaSuccess) {
        dense_free(d);
        return fail(PF_NO_MEMORY, "coarse dense solver: allocation of 3 x %d^2 doubles failed", d->np);
    }
    return PF_OK;
}

void dense_free(Dense* d) {
    if (d->M) cudaFree(d->M);
    if (d->Linv) cudaFree(d->Linv);
    if (d->Ainv) cudaFree(d->Ainv);
    if (d->fail) cudaFree(d->fail);
    d->M = d->Linv = d->Ainv = nullptr;
    d->fail = nullptr;
}

int dense_factor_linv(Dense* d, double beta, cudaStream_t st) {
    const int np = d->np, nt = np / TB;
    PF_CUDA(cudaMemsetAsync(d->fail, 0, sizeof(int), st));
    pf::count_launch();
    k_pad_diag<<<(np + 255) / 256, 256, 0, st>>>(d->M, d->n, np, beta);
    for (int p = 0; p < nt; p++) {
        pf::count_launch();
        k_potrf_tile<<<1, dim3(TB, TB), 0, st>>>(d->M, np, p, d->fail);
        if (p + 1 < nt) {
            pf::count_launch();
            k_trsm<<<nt - p - 1, TB, 0, st>>>(d->M, np, p);
            const int T = nt - p - 1;
            pf::count_launch();
            k_syrk<<<T * (T + 1) / 2, dim3(TB, TB), 0, st>>>(d->M, np, p);
        }
    }
    PF_CUDA(cudaMemsetAsync(d->Linv, 0, (size_t)np * np * sizeof(double), st));
    pf::count_launch();
    k_trtri_tiles<<<nt, TB, 0, st>>>(d->M, d->Linv, np);
    for (int i = 1; i < nt; i++) {
        pf::count_launch();
        k_linv_row<<<i, dim3(TB, TB), 0, st>>>(d->M, d->Linv, np, i);
    }
    PF_LAUNCH_CHECK("dense factorisation launch");
    return PF_OK;
}

int dense_factor_invert(Dense* d, double beta, cudaStream_t st) {
    int s = dense_factor_linv(d, beta, st);
    if (s) return s;
    const int np = d->np, nt = np / TB;
    pf::count_launch();
    k_ainv<<<dim3(nt, nt), dim3(TB, TB), 0, st>>>(d->Linv, d->Ainv, np, nt);
    PF_LAUNCH_CHECK("coarse factorisation launch");
    return PF_OK;
}

template <typename T>
int dense_solve(const Dense* d, const T* b, T* x, const int* skip, cudaStream_t st) {
    pf::count_launch();
    PF_CUDA(launch_pdl(k_dense_matvec<T>, dim3((d->n + 7) / 8), dim3(256), 0, st, (const double*)d->Ainv, d->np, d->n, b,
                       x, skip));
    PF_LAUNCH_CHECK("coarse solve launch");
    return PF_OK;
}
template int dense_solve<double>(const Dense*, const double*, double*, const int*, cudaStream_t);
template int dense_solve<float>(const Dense*, const float*, float*, const int*, cudaStream_t);

}  // namespace pf
