// Element operator object and the launchers other translation units use.
#pragma once

#include "common.cuh"

// corner l of an element sits at (kCXd(l), kCYd(l), kCZd(l)) relative to its lowest node,
// in the reference local order (pyFANTOM/physics/LinearElasticity.py:776-784 node signs).
__host__ __device__ __forceinline__ int kCXd(int l) { return (0x66 >> l) & 1; }
__host__ __device__ __forceinline__ int kCYd(int l) { return (0xCC >> l) & 1; }
__host__ __device__ __forceinline__ int kCZd(int l) { return (0xF0 >> l) & 1; }

struct pf_op {
    pf::Grid grid;
    double K0[24 * 24];  // row-major element matrix (8x8 used in 2D)
    double blk[8][3][3]; // Walsh-class blocks of K0 (4 classes of 2x2 in 2D)
};

namespace pf {

using Op = pf_op;

int op_factorise(Op* op);

template <typename T, typename TE>
int launch_fine_matvec(const Op* op, const TE* E, const T* u, const uint8_t* mask, const Epi<T>& epi,
                       cudaStream_t st);
long long fine_matvec_num_blocks(const Op* op, int fp32);

template <typename T>
int launch_diagonal(const Op* op, const double* E, const uint8_t* mask, T* diag, cudaStream_t st);
int launch_sensitivity(const Op* op, const double* U, double* dk, cudaStream_t st);
int launch_adjoint(const Op* op, const double* U, const double* rho, const pf_simp_params& P, double scale,
                   double* out, cudaStream_t st);
int launch_pack_mask(const Op* op, const uint8_t* con, uint8_t* mask, cudaStream_t st);

}  // namespace pf
