/*
 * pyfantom_b200.h -- C ABI of the B200 (sm_100a) structured SIMP / MGCG library.
 *
 * The library replaces the CuPy RawModule kernels and launch wrappers of the reference
 * pyFANTOM CUDA backend for structured Q4 / H8 meshes.  Every entry point returns an int
 * status (PF_OK = 0); on failure pf_last_error() holds a message.  Pointers are DEVICE
 * pointers unless the name starts with h_.  `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream).  No entry point allocates device memory except the
 * *_create functions, which own what they allocate until the matching *_destroy.
 *
 * Layouts (reference pyFANTOM/core/CUDA/Kernels/_geom.py:23-49):
 *   3D node (i,j,k) -> k + nz*(i + nx*j) ; element (i,j,k) -> (i*nely + j)*nelz + k
 *   2D node (i,j)   -> i + nx*j          ; element (i,j)   -> i*nely + j
 *   vectors are interleaved by DOF: v[node*dof + d]  (dof = dim)
 *   node_mask: one uint8 per node, bit d set = DOF d is a Dirichlet DOF (NULL = none)
 *   block stencils (coarse operators): structure-of-arrays
 *     A[((nb*dof + a)*dof + b)*n_nodes + node], nb = (dx+1) + 3(dy+1) [+ 9(dz+1)],
 *     i.e. the same 27 (3D) / 9 (2D) dof x dof blocks per row, in the same order, as the
 *     reference's padded CSR (pyFANTOM/core/CUDA/Kernels/mgm.cu:384-395).
 */
#ifndef PYFANTOM_B200_H
#define PYFANTOM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum pf_status {
    PF_OK = 0,
    PF_NOT_CONVERGED = 1, /* maxiter reached before the tolerance */
    PF_BREAKDOWN = 2,     /* p.Kp <= 0 or r.z <= 0 in PCG (operator not SPD on the iterate) */
    PF_NONFINITE = 3,     /* NaN / Inf found in an input or an iterate */
    PF_TIMEOUT = 4,       /* a bounded device-side wait gave up */
    PF_BAD_ARG = 5,       /* invalid argument (sizes, NULL pointers, unsupported options) */
    PF_CUDA_ERROR = 6,    /* a CUDA runtime call failed */
    PF_NO_MEMORY = 7,     /* device allocation failed */
    PF_UNSUPPORTED = 8,   /* valid input the library does not handle (e.g. K0 without
                             axis-reflection symmetry) */
    PF_FACTOR_FAILED = 9  /* coarse Cholesky hit a non-positive pivot */
};

typedef struct pf_grid {
    int dim;    /* 2 or 3 */
    int nel[3]; /* elements along x, y, z (nel[2] ignored in 2D) */
} pf_grid;

/* ---- library ------------------------------------------------------------------------ */
int pf_version(void);                     /* 100*major + minor */
unsigned long long pf_launch_count(void);  /* kernels launched by this library so far */
const char* pf_last_error(void);          /* message of the last failure on this thread */
const char* pf_status_string(int status); /* static name of a status code */

/* ---- element operator (replaces the K_single + node-incidence state of
 *      pyFANTOM/stiffness/CUDA/_FEA.py:326-366) --------------------------------------- */
typedef struct pf_op pf_op;
/* h_K0: host row-major element matrix (24x24 for H8, 8x8 for Q4), DOF order (node, comp)
 * with the reference local node order.  Fails with PF_UNSUPPORTED if K0 is not invariant
 * under the element's axis reflections (the block structure the kernels rely on). */
int pf_op_create(const pf_grid* grid, const double* h_K0, pf_op** out);
int pf_op_destroy(pf_op* op);
/* Which FP32 fine matvec serves cube elements: 0 = one element per thread (default, the
 * kernel of the other element shapes as well), 1 = two z-neighbouring elements per thread
 * in packed FP32 arithmetic (half the shuffles and row exchanges per element, but twice the
 * registers: one block of 12 warps per SM; 137 us against 78 us for variant 0 at
 * 256x128x128 on a B200).  Set it before creating solvers on the operator. */
int pf_op_set_variant(pf_op* op, int variant);
/* node mask from a per-DOF bool array (pyFANTOM/stiffness/CUDA/_FEA.py:441-456) */
int pf_pack_mask(const pf_op* op, const uint8_t* con_dof, uint8_t* node_mask, void* stream);
/* Explicit CSR of the matrix the matvec applies, Z K(E) Z + (I - Z) (StructuredStiffnessKernel.
 * construct, pyFANTOM/stiffness/CUDA/_FEA.py:484-516): row_ptr [n_dof + 1], col and val
 * [pf_csr_nnz(op)], int32 indices, columns increasing within a row; the pattern depends on
 * the grid only (couplings of constrained DOFs are stored as zeros).  PF_UNSUPPORTED when
 * the nonzeros exceed 32-bit indices. */
long long pf_csr_nnz(const pf_op* op);
int pf_construct_csr_f64(const pf_op* op, const double* E, const uint8_t* node_mask, int* row_ptr, int* col,
                         double* val, void* stream);

/* y = K(E) u with Dirichlet identity rows: y_c = u_c at constrained DOFs, constrained
 * columns skipped.  Replaces mat_vec_node_basis_parallel[_wcon]_cuda_kernel
 * (pyFANTOM/core/CUDA/Kernels/matvec.cu:1-98) behind StructuredStiffnessKernel._matvec
 * (pyFANTOM/stiffness/CUDA/_FEA.py:518-549). */
int pf_matvec_f64(const pf_op* op, const double* E, const double* u, const uint8_t* node_mask,
                  double* y, void* stream);
int pf_matvec_f32(const pf_op* op, const float* E, const float* u, const uint8_t* node_mask,
                  float* y, void* stream);
/* FP32 matvec with the element scales stored as BF16 (bit patterns, round-to-nearest of the
 * FP64 E): the V-cycle operator of the mixed form with BF16 density storage. */
int pf_matvec_f32_bf16(const pf_op* op, const uint16_t* E_bf16, const float* u, const uint8_t* node_mask,
                       float* y, void* stream);
/* diag(K(E)), 1 at constrained DOFs.  Replaces get_diagonal_node_basis_cuda_kernel
 * (diag.cu:1-47) behind StructuredStiffnessKernel.diagonal (_FEA.py:368-420). */
int pf_diagonal_f64(const pf_op* op, const double* E, const uint8_t* node_mask, double* d,
                    void* stream);
/* dk_e = -u_e^T K0 u_e.  Replaces process_dk_kernel_cuda (grad.cu:1-16) behind
 * StructuredStiffnessKernel.process_grad (_FEA.py:458-482). */
int pf_sensitivity_f64(const pf_op* op, const double* U, double* dk, void* stream);

/* ---- grid transfers (restriction_3d/2d_kernel, prolongation_3d/2d_kernel,
 *      pyFANTOM/core/CUDA/Kernels/mgm.cu:1-244, via core/CUDA/_mgm.py:173-264) ---------- */
/* `fine` is the fine grid (at least 2 elements per axis); the coarse grid has floor(nel/2)
 * elements per axis, as the reference's (core/CUDA/_mgm.py:24-27). */
int pf_restrict_f64(const pf_grid* fine, const double* vf, double* vc, void* stream);
int pf_prolong_f64(const pf_grid* fine, const double* vc, double* vf, void* stream);

/* ---- Galerkin coarse operators (get_restricted_3d/2d_l0/l1p_nnz_based,
 *      mgm.cu:247-895, via core/CUDA/_mgm.py:19-171) ---------------------------------- */
int pf_galerkin_l0_f64(const pf_op* op, const double* E, const uint8_t* node_mask, double* A_coarse,
                       void* stream);
int pf_galerkin_l1p_f64(const pf_grid* fine, const double* A_fine, double* A_coarse, void* stream);
int pf_stencil_matvec_f64(const pf_grid* grid, const double* A, const double* u, double* y,
                          void* stream);
size_t pf_stencil_size(const pf_grid* grid); /* doubles in one block stencil of `grid` */

/* ---- multigrid-preconditioned CG (MultiGrid, pyFANTOM/solvers/CUDA/_solvers.py:330-660) */
typedef struct pf_mg pf_mg;
typedef struct pf_mg_config {
    int n_level;        /* coarse levels below the fine grid (reference n_level) */
    int n_smooth;       /* damped-Jacobi sweeps before and after the coarse correction */
    double omega;       /* reference omega (max omega of the adaptive schedule) */
    double min_omega;   /* reference min_omega argument (effective = max(omega/2, min_omega)) */
    double omega_boost; /* omega growth per level (reference uses 1.06) */
    double coarse_beta; /* diagonal shift of the coarse Cholesky (CHOLMOD beta = 1e-6) */
    int precision;      /* 0 = FP64 V-cycle, 1 = FP32 V-cycle inside FP64 CG,
                           2 = FP32 V-cycle reading BF16 element scales, inside FP64 CG */
    int check_every;    /* host convergence poll interval in iterations (>= 1) */
    int coarse_op;      /* 0 = level 1 applied element by element from the fine densities when
                           K0 is an isotropic box element and level 1 is smoothed (else its
                           stencil); 1 = assembled stencils on every level */
    unsigned w_mask;    /* bit l set: level l repeats its coarse correction from the updated
                           iterate (the reference's lower-case 'w' cycle at the levels in
                           w_level, _solvers.py:550-569); 0 = V-cycle */
    double omega_fixed; /* 0: the reference's Jacobi weight schedule (min_omega at the start,
                           then min + (omega - min) / 2 exp(-500 (clip(R, tol, 0.1) - tol)));
                           > 0: this weight in every V-cycle of the solve, a fixed
                           preconditioner (no reference counterpart) */
} pf_mg_config;

typedef struct pf_solve_info {
    int iterations;     /* PCG iterations performed */
    int status;         /* pf_status of the solve */
    double residual;    /* ||r|| / ||b|| of the recursive residual at exit */
    double setup_ms;    /* device time of the hierarchy setup inside this call */
    double solve_ms;    /* device time of the iterations */
} pf_solve_info;

int pf_mg_create(const pf_op* op, const pf_mg_config* cfg, pf_mg** out);
int pf_mg_destroy(pf_mg* mg);
/* Build D^-1, the Galerkin hierarchy and the coarse factor for densities E
 * (MultiGrid._setup, _solvers.py:442-516). */
int pf_mg_setup(pf_mg* mg, const double* E, const uint8_t* node_mask, void* stream);
/* z = V-cycle(r) (W-cycle at the levels of cfg.w_mask) from a zero initial guess with
 * Jacobi weight omega (MultiGrid._multi_grid, _solvers.py:518-571). */
int pf_mg_vcycle(pf_mg* mg, const double* r, double* z, double omega, void* stream);
/* PCG on K(E) x = b preconditioned by the V-cycle (MultiGrid.solve, _solvers.py:573-660).
 * Requires pf_mg_setup.  use_x0 != 0 starts from the contents of x, else from 0.
 * Blocks the calling thread until the solve ends; info is filled on return. */
int pf_mg_solve(pf_mg* mg, const double* b, double* x, int use_x0, double tol, int maxiter,
                pf_solve_info* info, void* stream);
/* Deflation space of the following pf_mg_solve calls (a learned coarse-grid correction): Q =
 * the three displacement components of the nodal field y (n DOFs, zero at constrained DOFs),
 * W = K Q.  PCG starts from x0 = x + Q G^-1 Q^T (b - K x), G = Q^T W, and removes
 * Q G^-1 W^T z from each preconditioned residual z (deflated PCG of Saad, Yeung, Erhel and
 * Guyomarc'h, SIAM J. Sci. Comput. 21 (2000)); the V-cycle is unchanged.  Components whose
 * G diagonal is zero are left out.  Requires pf_mg_setup; each pf_mg_setup clears it (K Q
 * changes with the densities).  y = NULL clears it.  No reference counterpart: the
 * reference's MultiGrid.solve (_solvers.py:573-660) has no coarse-space deflation. */
int pf_mg_set_deflation(pf_mg* mg, const double* y, void* stream);
/* y = A_l u with the operator the V-cycle applies on level l in [0, n_level) (l = 0: the
 * fine matvec; l = 1: the element-level operator or the stencil; deeper: the stencil), in
 * the V-cycle precision (double for precision 0, float otherwise).  Requires pf_mg_setup. */
int pf_mg_level_matvec(pf_mg* mg, int level, const void* u, void* y, void* stream);
/* h_elem_level1 = 1 if level 1 is applied element by element; h_dirty = its number of
 * coarse elements with an explicit matrix (those touching a constraint). */
int pf_mg_level_info(const pf_mg* mg, int* h_elem_level1, int* h_dirty);
/* Diagnostics: time every fine-level matvec launch of the following solves with CUDA
 * events (at most max_launches per solve; 0 disables), and read the last solve's totals:
 * device milliseconds, launches, and algorithmic bytes (each operand counted once). */
int pf_mg_set_profiling(pf_mg* mg, int max_launches);
int pf_mg_profile(const pf_mg* mg, double* h_ms, long long* h_launches, double* h_bytes);
/* Which fine-level matvec launches the profiling records: 1 = the FP64 ones (PCG matvec,
 * FP64 V-cycle), 2 = the FP32 ones (V-cycle of the mixed forms), 3 = both (default). */
int pf_mg_profile_select(pf_mg* mg, int which);
/* Number of doubles of device workspace pf_cg_solve needs for `op`. */
size_t pf_cg_workspace_size(const pf_op* op);
/* Unpreconditioned CG on K(E) x = b (the matrix-free CG of _solvers.py:22-132).  `work`
 * holds pf_cg_workspace_size(op) doubles. */
int pf_cg_solve(const pf_op* op, const double* E, const uint8_t* node_mask, const double* b, double* x,
                int use_x0, double tol, int maxiter, double* work, pf_solve_info* info, void* stream);

/* ---- density filter (CuStructuredFilter2D/3D, pyFANTOM/geom/CUDA/_filters.py:14-201,
 *      kernels filters.cu:1-154) ------------------------------------------------------ */
typedef struct pf_filter pf_filter;
/* h_offsets: n_taps x dim ints, h_weights: n_taps doubles (normalised to sum 1) */
int pf_filter_create(const pf_grid* grid, int n_taps, const int* h_offsets, const double* h_weights,
                     pf_filter** out);
int pf_filter_destroy(pf_filter* f);
int pf_filter_normalizer_f64(const pf_filter* f, double* out, void* stream);
int pf_filter_fwd_f64(const pf_filter* f, const double* x, double* y, void* stream);
int pf_filter_adj_f64(const pf_filter* f, const double* x, double* y, void* stream);

/* ---- SIMP element-wise steps (MinimumCompliance.penalize / penalize_grad,
 *      pyFANTOM/Problem/CUDA/MinimumCompliance.py:305-367) ----------------------------- */
typedef struct pf_simp_params {
    double penalty;
    double void_value;
    double E_mul;
    double beta; /* Heaviside sharpness (used when heavyside != 0) */
    double eta;  /* Heaviside threshold */
    int heavyside;
} pf_simp_params;
/* E = penalize(rho); dE = penalize_grad(rho) (either output may be NULL) */
int pf_penalize_f64(long long n, const double* rho, const pf_simp_params* p, double* E, double* dE,
                    void* stream);
/* Fused adjoint of the compliance (self-adjoint: the adjoint state is -U):
 * out_e = scale * dE/drho(rho_e) * (-u_e^T K0 u_e), dE/drho as pf_penalize_f64's dE, rho
 * the filtered densities.  dc/dx = H^T out (pf_filter_adj_f64).  Replaces the chain
 * process_grad -> penalize_grad -> product of MinimumCompliance._compute
 * (pyFANTOM/Problem/CUDA/MinimumCompliance.py:428-438) with one kernel. */
int pf_adjoint_f64(const pf_op* op, const double* U, const double* rho, const pf_simp_params* p,
                   double scale, double* out, void* stream);
/* out_e = dE_e * dk_e  (the element factor of the compliance sensitivity) */
int pf_mul_f64(long long n, const double* a, const double* b, double* out, void* stream);

/* ---- reductions --------------------------------------------------------------------- */
size_t pf_dot_workspace_size(long long n); /* doubles */
/* *result (device) = a . b, deterministic order; work holds pf_dot_workspace_size(n) doubles */
int pf_dot_f64(long long n, const double* a, const double* b, double* result, double* work, void* stream);

/* ---- OC update (Optimizers/CUDA/OC.py:67-144, single constraint) ---------------------- */
size_t pf_oc_workspace_size(long long n); /* doubles */
/* One OC step: ocP = x sqrt(max(-df/dg, 0)) (1e-3 everywhere if all zero), bisection on
 * lambda in [1e-9, 1e9] until (l2-l1)/(l2+l1) <= 1e-8 testing dg.x_new - vf <= 0,
 * x_new = max(0, max(x-move, min(1, min(x+move, ocP/lambda)))) (bounds clipped to [0,1]).
 * h_out (host, may be NULL) receives {change = ||x_new - x||_2, lambda, steps}.
 * work holds pf_oc_workspace_size(n) doubles. */
int pf_oc_update_f64(long long n, const double* x, const double* df, const double* dg, double vf,
                     double move, double* x_new, double* work, double* h_out, void* stream);

/* ---- learned warm start: kernels of a small 3D convolutional network ---------------
 * No counterpart in the reference (the learned form of this library).  float32
 * activations [N][C][X][Y][Z], weights [Cout][Cin][3][3][3], zero padding 1, stride 1|2
 * (output extent (n-1)/stride + 1).  relu != 0 fuses max(0, .) into the forward. */
int pf_cnn_conv3d_fwd_f32(const float* x, int N, int Cin, int X, int Y, int Z, const float* w, const float* b,
                          int Cout, int stride, int relu, float* y, void* stream);
/* dx = W^T dy (accumulate != 0: dx += W^T dy) */
int pf_cnn_conv3d_bwd_data_f32(const float* dy, int N, int Cin, int X, int Y, int Z, const float* w, int Cout,
                               int stride, int accumulate, float* dx, void* stream);
/* The forward and the input gradient on the tensor cores (tcgen05.mma implicit GEMM): same
 * arguments and layouts as the FP32 versions, operands rounded to BF16, accumulation in
 * FP32; at most 256 output channels.  err (device int, set to 0 by the caller) becomes 1 if
 * a wait for the tensor cores ran out (the output is then not written). */
int pf_cnn_conv3d_fwd_tc(const float* x, int N, int Cin, int X, int Y, int Z, const float* w, const float* b,
                         int Cout, int stride, int relu, float* y, int* err, void* stream);
int pf_cnn_conv3d_bwd_data_tc(const float* dy, int N, int Cin, int X, int Y, int Z, const float* w, int Cout,
                              int stride, int accumulate, float* dx, int* err, void* stream);
/* dw, db on the tensor cores (BF16 operands, FP32 accumulation; the voxels are split into
 * fixed ranges whose partial sums are added in order).  work: the number of floats
 * pf_cnn_conv3d_bwd_weight_tc_workspace returns for these sizes; db may be NULL. */
size_t pf_cnn_conv3d_bwd_weight_tc_workspace(int N, int Cin, int X, int Y, int Z, int Cout, int stride);
int pf_cnn_conv3d_bwd_weight_tc(const float* x, const float* dy, int N, int Cin, int X, int Y, int Z, int Cout,
                                int stride, float* dw, float* db, float* work, int* err, void* stream);
size_t pf_cnn_conv3d_bwd_weight_workspace(int Cin, int Cout); /* floats */
int pf_cnn_conv3d_bwd_weight_f32(const float* x, const float* dy, int N, int Cin, int X, int Y, int Z, int Cout,
                                 int stride, float* dw, float* db, float* work, void* stream);
int pf_cnn_relu_bwd_f32(long long n, const float* y, float* dy, void* stream); /* dy *= (y > 0) */
/* nearest 2x upsampling of NC channels of X x Y x Z (backward: x = dy fine, y = dx coarse) */
int pf_cnn_upsample2_f32(int NC, int X, int Y, int Z, const float* x, float* y, int backward, void* stream);
/* dst[n][c_off + c] (+)= src[n][c] for c < Csrc; gather != 0 copies the other way */
int pf_cnn_copy_channels_f32(int N, int Csrc, long long V, const float* src, int Cdst, int c_off, int accumulate,
                             int gather, float* dst, void* stream);
/* out[n][c] = scale * sum_v src[n][c_off + c][v] (src has Csrc channels of V voxels) */
int pf_cnn_channel_sum_f32(int N, int C, long long V, const float* src, int Csrc, int c_off, float scale, float* out,
                           void* stream);
/* dst[n][c_off + c][v] (+)= scale * g[n][c] for every voxel v (dst has Cdst channels) */
int pf_cnn_channel_bcast_f32(int N, int C, long long V, const float* g, float scale, int Cdst, int c_off,
                             int accumulate, float* dst, void* stream);
/* cells [N][3][X][Y][Z] -> nodal 3-vectors [N][nodes][3] (mean of adjacent cells), or back */
int pf_cnn_cell2node_f32(int N, int X, int Y, int Z, const float* in, float* out, int backward, void* stream);
size_t pf_cnn_mse_workspace(long long n); /* doubles */
/* loss = mean((pred - target)^2) into the device double *loss; grad (may be NULL) = d loss / d pred */
int pf_cnn_mse_f32(long long n, const float* pred, const float* target, float* grad, double* loss, double* work,
                   void* stream);
/* one bias-corrected Adam step (step counts from 1) */
int pf_cnn_adam_f32(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                    float eps, int step, void* stream);
/* Network input of one sample on the cell grid fine->nel / P (every count divisible by P):
 * out [8][X/P][Y/P][Z/P] = E^(1/3) of the block-mean stiffness; nodal forces of the
 * block's closed node box (shared nodes split between blocks) divided by max|f|; the
 * constrained fraction of the 24 DOFs at the cell corners; cell-centre coordinates
 * scaled to (-1, 1).  E [elements], f [dof] device doubles, node_mask from pf_pack_mask
 * (NULL: unconstrained), work: 1 unsigned. */
int pf_cnn_features_f32(const pf_grid* fine, int P, const double* E, const double* f, const uint8_t* node_mask,
                        unsigned* work, float* out, void* stream);
/* x0 [dof] = trilinear interpolation onto the fine mesh of the nodal field coarse_nodes
 * [(X/P+1)(Y/P+1)(Z/P+1)][3] of the mesh with nel / P elements; 0 on constrained DOFs. */
int pf_cnn_guess_f64(const pf_grid* fine, int P, const float* coarse_nodes, const uint8_t* node_mask, double* x0,
                     void* stream);
/* x0 *= alpha = (x0.b) / (x0.Kx0) (0 if x0.Kx0 <= 0); work: pf_cnn_energy_scale_workspace()
 * doubles; work[size - 2] = alpha, work[size - 1] = ||b - alpha Kx0|| / ||b||. */
size_t pf_cnn_energy_scale_workspace(void);
int pf_cnn_energy_scale_f64(long long n, double* x0, const double* Kx0, const double* b, double* work, void* stream);
/* Of two initial guesses xa, xb of K u = f (with Kxa, Kxb their products), write to out the
 * one whose energy-optimal multiple alpha x (alpha = x.f / x.Kx) has the lower energy
 * -(x.f)^2 / (2 x.Kx), i.e. the smaller energy-norm error; a guess with x.Kx <= 0 counts as
 * the zero start.  out may alias xa or xb.  work: pf_cnn_guess_select_workspace() doubles;
 * its last four hold {alpha, choice (0 = xa, 1 = xb), energy of xa, energy of xb}. */
size_t pf_cnn_guess_select_workspace(void);
int pf_cnn_guess_select_f64(long long n, const double* xa, const double* Kxa, const double* xb, const double* Kxb,
                            const double* f, double* out, double* work, void* stream);

/* Energy-deficit training loss of a nodal prediction y for K u = b (y zero on constrained
 * DOFs, Ky = K y, c = b.u > 0): loss = 1 - (b.y)^2 / ((y.Ky) c), the relative energy
 * error left after scaling y by (b.y)/(y.Ky); grad [n] float = d loss / d y.
 * work: pf_cnn_energy_loss_workspace() doubles. */
size_t pf_cnn_energy_loss_workspace(void);
int pf_cnn_energy_loss_f64(long long n, const double* y, const double* Ky, const double* b, double c, float* grad,
                           double* loss, double* work, void* stream);

/* ---- direct solve for small problems (the reference's SPSOLVE,
 * solvers/CUDA/_solvers.py:245-328 with StructuredStiffnessKernel.construct,
 * stiffness/CUDA/_FEA.py:484-516): dense assembly of the free-DOF block of K(E), tiled
 * Cholesky and inverse factor, x = L^-T L^-1 b; constrained entries of x are b's.
 * free_dofs [n_free] and dof_to_free [dof] (-1 when constrained) are int32 device
 * arrays; n_free <= 20480. */
typedef struct pf_direct pf_direct;
int pf_direct_create(const pf_op* op, pf_direct** out);
int pf_direct_destroy(pf_direct* d);
int pf_direct_solve_f64(pf_direct* d, const double* E, const int* free_dofs, const int* dof_to_free, int n_free,
                        const double* b, double* x, void* stream);

/* ---- multi-material SIMP (pyFANTOM/Problem/CUDA/MinimumCompliance.py:326-349,369-411) */
/* E[e] = max(sum_i E_mul_i a_i prod_{j!=i} (1 - a_j), void), a_i = H(rho_i)^p, and
 * dE[k][e] = dE/drho_k; rho and dE material-major [nm][ne]; 2 <= nm <= 8; h_E_mul host. */
int pf_penalize_multi_f64(long long ne, int nm, const double* rho, const pf_simp_params* p, const double* h_E_mul,
                          double* E, double* dE, void* stream);
/* OC with one volume constraint per material (variables material-major, dg the per-variable
 * constraint gradient, h_vf host [nm]): the multipliers are bisected in lockstep until all
 * meet the stopping rule (Optimizers/CUDA/OC.py:104-127).  h_out as pf_oc_update_f64
 * (lambda and steps of material 0). */
size_t pf_oc_multi_workspace_size(long long ne, int nm);
int pf_oc_update_multi_f64(long long ne, int nm, const double* x, const double* df, const double* dg,
                           const double* h_vf, double move, double* x_new, double* work, double* h_out, void* stream);

/* ---- PGD (pyFANTOM/Optimizers/CUDA/PGD.py:6-372) --------------------------------------- */
size_t pf_pgd_workspace_size(long long n); /* doubles, for the stats, step and single projection */
/* h_out[8] (host) = {df.df, max|df|, df.df_last, df_last.df_last, s.y, s.s, y.y, max|y|}
 * with s = x_last - x, y = df_last - df (PGD.alpha, :107-142); x_last, df_last may both
 * be NULL (first iteration: entries 2..7 are 0). */
int pf_pgd_stats_f64(long long n, const double* x, const double* df, const double* x_last, const double* df_last,
                     double* work, double* h_out, void* stream);
/* d = -df + beta d_last (d_last NULL: d = -df), x_new = x + alpha d (PGD.iter, :226-236) */
int pf_pgd_step_f64(long long n, const double* x, const double* df, const double* d_last, double beta, double alpha,
                    double* d, double* x_new, void* stream);
/* x_new = clip(xs + l dg, lo, hi) with l from the reference bisection on dg.x - vf <= 0
 * (project_to_feasible, :144-170: l in [-1e12, 0], midpoint rule, stop when
 * (l2-l1)/(l2+l1) <= tol, l = 0 when clip(xs) is feasible).  h_out (host, may be NULL)
 * = {l, bisection steps, feasible at l = 0}. */
int pf_pgd_project_f64(long long n, const double* xs, const double* dg, double vf, double lo, double hi, double tol,
                       double* x_new, double* work, double* h_out, void* stream);
/* The same projection for one volume constraint per block of the design
 * (project_to_feasible, :146-170 with m = nm > 1, the independent-constraints branch that
 * MinimumCompliance takes for nm materials).  xs, x_new: nm blocks of ne; dg: nm blocks of
 * ne, block c = row c of the constraint gradient on block c (MinimumCompliance's rows are
 * zero elsewhere); h_vf (host): nm volume fractions.  The nm bisections run in lockstep
 * while any block is unconverged (a block feasible at l = 0 keeps bisecting towards zero,
 * about 1100 sweeps).  h_out (host, required) = {sweeps, feasible at l = 0 in every block,
 * l_0 .. l_{nm-1}}.  1 <= nm <= 8; work: pf_pgd_multi_workspace_size(ne, nm) doubles. */
size_t pf_pgd_multi_workspace_size(long long ne, int nm);
int pf_pgd_project_multi_f64(long long ne, int nm, const double* xs, const double* dg, const double* h_vf, double lo,
                             double hi, double tol, double* x_new, double* work, double* h_out, void* stream);

/* ---- OC update without allocation --------------------------------------------------
 * No counterpart in the reference.  Same computation and outputs as pf_oc_update_f64,
 * for callers that cannot allocate device memory where they run the OC step: plugins
 * inside a framework that owns the device memory (its caching allocator may hold nearly
 * all of it, and the plugin must not allocate behind its back) and per-iteration
 * callbacks with a latency budget (cudaMalloc synchronises the device).  The scratch is
 * a static device array of the library sized for PF_OC_NOALLOC_MAX_ELEMS elements
 * (16.9 MB held by every GPU that loads the library until the process exits).  Larger n
 * is rejected with PF_BAD_ARG.  The first call on each device resolves the array's
 * address with that device current and keeps it (it may also load the library's device
 * code); after a cudaDeviceReset the kept address is stale and the entry point must not
 * be called again in that process.  A non-NULL h_out makes the call wait for the stream to deliver
 * {||x_new - x||, lambda, steps}; pass NULL where the caller must not wait.  Calls share
 * the array: calls that overlap on the GPU race. */
#define PF_OC_NOALLOC_MAX_ELEMS 2097152
int pf_oc_update_noalloc_f64(long long n, const double* x, const double* df, const double* dg, double vf,
                             double move, double* x_new, double* h_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PYFANTOM_B200_H */
