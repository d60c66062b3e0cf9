// Launchers of the multigrid level kernels (mgkern.cu) and the dense coarse solver (dense.cu).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace pf {

// optional fused first Jacobi sweep of the coarse level: x = omega * scale * dinv * b_c
template <typename T>
struct Jacobi0 {
    T* x = nullptr;
    const T* dinv = nullptr;
    const double* omega = nullptr;
    double scale = 1.0;
};
template <typename TI, typename TO>
int launch_restrict(const Grid& gf, const TI* vf, TO* vc, const int* skip, cudaStream_t st,
                    Jacobi0<TO> j0 = Jacobi0<TO>());
template <typename T>
int launch_prolong(const Grid& gf, const T* vc, T* vf, const int* skip, cudaStream_t st);
// half = true: A is the half storage of launch_stencil_half (centre and upper offsets, in
// tiles of 32 nodes)
template <typename T>
int launch_stencil_matvec(const Grid& g, const T* A, const T* u, const Epi<T>& epi, cudaStream_t st,
                          bool half = false);
long long stencil_half_size(const Grid& g);  // elements of the half storage
template <typename T>
int launch_stencil_half(const Grid& g, const double* A, T* H, cudaStream_t st);
long long stencil_matvec_num_blocks(const Grid& g);

void galerkin_child_matrices(int dim, const double* K0, double* Kc);
int launch_coarse_flags(const Grid& gf, const uint8_t* mask, uint8_t* elem_flag, uint8_t* node_flag, cudaStream_t st);
int launch_galerkin_l0(const Grid& gf, const double* E, const uint8_t* mask, const uint8_t* elem_flag,
                       const uint8_t* node_flag, const double* K0_dev, const double* Kc_dev, double* A,
                       cudaStream_t st);
int launch_galerkin_l1p(const Grid& gf, const double* Af, double* Ac, cudaStream_t st);
// the same product as three one-axis passes (3D; 2D falls back to launch_galerkin_l1p);
// scratch holds galerkin_sep_scratch(gf) doubles
long long galerkin_sep_scratch(const Grid& gf);
int launch_galerkin_sep(const Grid& gf, const double* Af, double* Ac, double* scratch, cudaStream_t st);
template <typename T>
int launch_stencil_dinv(const Grid& g, const double* A, T* dinv, cudaStream_t st);
int launch_stencil_to_dense(const Grid& g, const double* A, double* M, long long ld, cudaStream_t st);
int launch_d2f(long long n, const double* a, float* b, cudaStream_t st);
// FP64 -> BF16 (round to nearest even)
int launch_d2bf(long long n, const double* a, __nv_bfloat16* b, cudaStream_t st);

// dense SPD coarse solver: factor (M + beta I) of order n (padded to a multiple of 32,
// ld = padded order) and form its inverse; x = inv * b.
struct Dense {
    int n = 0, np = 0;            // order and padded order
    double* M = nullptr;          // np x np work / factor
    double* Linv = nullptr;       // np x np inverse factor
    double* Ainv = nullptr;       // np x np inverse
    int* fail = nullptr;          // device flag: first failing pivot + 1
};
int dense_alloc(Dense* d, int n);
void dense_free(Dense* d);
// M must hold the matrix (rows/cols >= n zero) before the call
int dense_factor_invert(Dense* d, double beta, cudaStream_t st);
// factor and inverse factor only (Linv = L^-1); no explicit inverse
int dense_factor_linv(Dense* d, double beta, cudaStream_t st);
template <typename T>
int dense_solve(const Dense* d, const T* b, T* x, const int* skip, cudaStream_t st);

}  // namespace pf
