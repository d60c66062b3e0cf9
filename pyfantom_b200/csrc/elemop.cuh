// Element operator object and the launchers other translation units use.
#pragma once

#include "common.cuh"

// corner l of an element sits at (kCXd(l), kCYd(l), kCZd(l)) relative to its lowest node,
// in the reference local order (pyFANTOM/physics/LinearElasticity.py:776-784 node signs).
__host__ __device__ __forceinline__ int kCXd(int l) { return (0x66 >> l) & 1; }
__host__ __device__ __forceinline__ int kCYd(int l) { return (0xCC >> l) & 1; }
__host__ __device__ __forceinline__ int kCZd(int l) { return (0xF0 >> l) & 1; }

// value index (0..6) of sparse coefficient q (see pf_op::coef) for a cube element:
// class 0 a b b a b a | 1, 2 b c b | 3 d d d e | 4 b c b | 5, 6 d d d e | 7 f g g f g f
__host__ __device__ constexpr int cube_index(int q) {
    return q < 6 ? ((q == 0 || q == 3 || q == 5) ? 0 : 1)
                 : q < 12 ? ((q - 6) % 3 == 1 ? 2 : 1)
                 : q < 16 ? (q == 15 ? 4 : 3)
                 : q < 19 ? (q == 17 ? 2 : 1)
                 : q < 27 ? ((q == 22 || q == 26) ? 4 : 3)
                 : ((q == 27 || q == 30 || q == 32) ? 5 : 6);
}

struct pf_op {
    pf::Grid grid;
    double K0[24 * 24];  // row-major element matrix (8x8 used in 2D)
    double blk[8][3][3]; // Walsh-class blocks of K0 (4 classes of 2x2 in 2D)
    // 3D: the 33 distinct nonzeros of the class blocks when they have the sparsity of an
    // isotropic box element (sparse != 0), and the 7 values of a cube element (cube != 0)
    double coef[33];
    int sparse, cube;
    double cube_v[7];
    int variant;  // FP32 fine matvec of cube elements: 0 one element per lane, 1 two (packed)
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
