// Multigrid-preconditioned CG and plain CG on the structured stiffness operator.
//
// Algorithm (reference MultiGrid, pyFANTOM/solvers/CUDA/_solvers.py:437-660):
//   setup   D0^-1 = 1/diag(K(E)); A1 = R (Z K Z + I - Z) P; A_{l+1} = R A_l P;
//           coarsest: (A_L + beta I)^-1 on the device;
//   V-cycle from x = 0 at every level: n_smooth damped-Jacobi sweeps with
//           omega * boost^l, residual, restrict, recurse, prolong, n_smooth sweeps on
//           A e = r starting from the prolonged e, x += e;
//   PCG     omega starts at min_omega and after each iteration becomes
//           min_omega + (omega - min_omega)/2 * exp(-500 (clip(R, tol, 0.1) - tol))
//           (or stays at cfg.omega_fixed: a fixed preconditioner, no reference counterpart),
//           Fletcher-Reeves beta, stop when ||r||/||b|| < tol.
// Differences of form, not of result: every scalar (alpha, beta, omega, ||r||) lives in
// device memory and is consumed by the next kernel, so iterations are enqueued without
// host synchronisation; the host polls a completion flag every `check_every`
// iterations while the next chunk is already queued, and every kernel of an iteration
// past convergence returns immediately.  Jacobi sweeps, residuals, the final x += e and
// the r.z product are fused into the epilogues of the matvec kernels.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "coarse.cuh"
#include "common.cuh"
#include "elemop.cuh"
#include "mgkern.cuh"

namespace pf {

constexpr int kMaxLevel = 12;
constexpr int kRedThreads = 256;

struct PcgState {
    double rho_old, norm_b, alpha, beta, R, omega;
    double tol, min_omega, d_omega;
    int it, maxiter, done, status;
    int stop_le;  // 1: stop when R <= tol (cupyx cg, plain CG); 0: R < tol (MultiGrid)
    double coef[3];  // deflation: G^-1 Q^T r (start) or G^-1 W^T z (iterations)
};

struct Level {
    Grid g;
    long long ndof = 0;
    void* b = nullptr;  // right-hand side (level >= 1)
    void* x = nullptr;  // iterate / result
    void* t = nullptr;  // ping-pong partner
    void* r = nullptr;  // residual after pre-smoothing
    void* e = nullptr;  // coarse correction
    void* dinv = nullptr;
    double* A64 = nullptr;  // block stencil (level >= 1)
    void* H = nullptr;      // its half storage in the V-cycle precision (smoothed levels)
};

}  // namespace pf

struct pf_mg {
    const pf::Op* op = nullptr;
    pf_mg_config cfg;
    int fp32 = 0;
    int nlev = 0;
    pf::Level L[pf::kMaxLevel + 1];
    pf::Dense dense;
    double* K0_dev = nullptr;
    double* Kc_dev = nullptr;
    uint8_t* elem_flag = nullptr;
    uint8_t* node_flag = nullptr;
    const double* E = nullptr;
    const uint8_t* mask = nullptr;
    pf::CoarseOp* c1 = nullptr;     // element-level operator of level 1 (else its stencil)
    // deflation by a coarse space Q = [q_0 q_1 q_2], q_c = a field's component c (learned
    // coarse-grid correction): field, W = A Q (FP32) and G^-1 (FP64, 9 values + 3 flags)
    int defl = 0;
    float* yf = nullptr;
    double* Wd = nullptr;
    double* gscratch = nullptr;  // intermediate stencils of the separable Galerkin product (levels >= 2)
    double* dG = nullptr;
    float* Ef = nullptr;            // FP32 element scales of the V-cycle (precision 1)
    __nv_bfloat16* Eb = nullptr;    // BF16 element scales of the V-cycle (precision 2)
    double *r = nullptr, *p = nullptr, *q = nullptr;
    double* partials = nullptr;
    long long npartials = 0;
    pf::PcgState* st = nullptr;
    pf::PcgState* h_snap = nullptr;  // pinned, 2 snapshots
    cudaEvent_t ev[6] = {};  // 0,1 setup; 2 solve start; 3,4 chunk polls; 5 solve end
    bool ready = false;
    double setup_ms = 0.0;
    // optional CUDA-event timing of every fine-level matvec launch of a solve
    // internal copies that keep the pointers captured in the CUDA graphs valid across solves
    double* Eint = nullptr;
    double* bi = nullptr;
    double* xi = nullptr;
    cudaStream_t cs = nullptr;        // private stream the solve runs (and is captured) on
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t g_start[2] = {nullptr, nullptr};  // start sequence, without / with x0
    cudaGraphExec_t g_chunk = nullptr;                // check_every PCG iterations
    unsigned long long g_start_nodes[2] = {0, 0}, g_chunk_nodes = 0;
    const uint8_t* g_mask = nullptr;  // node mask the graphs were captured with
    int profile = 0;
    int profile_which = 3;         // bit 0: FP64 fine matvec launches, bit 1: FP32 ones
    std::vector<cudaEvent_t> pev;  // pairs (start, end)
    std::vector<double> pbytes;    // algorithmic bytes of each recorded launch
    int pn = 0;
    double prof_ms = 0.0, prof_bytes = 0.0;
    long long prof_launches = 0;
};

namespace pf {

// ---------------------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_jacobi0(long long n, const T* __restrict__ b, const T* __restrict__ dinv, const double* omega,
                          double scale, T* __restrict__ x, const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (skip && *skip) return;
    const T w = (T)((*omega) * scale);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = w * dinv[i] * b[i];
}

template <typename T>
__global__ void k_recip(long long n, T* v) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = T(1) / v[i];
}

__global__ void k_d2f_skip(long long n, const double* __restrict__ a, float* __restrict__ b, const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (skip && *skip) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// partial dot a.b per block (grid-stride), TB = type of b
template <typename TB>
__global__ void __launch_bounds__(kRedThreads) k_dot_partial(long long n, const double* __restrict__ a,
                                                             const TB* __restrict__ b, double* partials,
                                                             const int* skip) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (skip && *skip) return;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += a[i] * (double)b[i];
    s = block_sum<kRedThreads>(s, s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__device__ double sum_partials(const double* partials, long long np, double* s_red) {
    double s = 0.0;
    for (long long i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    return block_sum<kRedThreads>(s, s_red);
}

__device__ void defl_coef(const double* partials, long long np, int off, const double* dG, PcgState* st,
                          double* s_red);

__global__ void __launch_bounds__(kRedThreads) k_pcg_normb(const double* partials, long long np, PcgState* st) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    const double bb = sum_partials(partials, np, s_red);
    if (threadIdx.x == 0) {
        st->norm_b = sqrt(bb);
        st->it = 0;
        st->done = 0;
        st->status = PF_NOT_CONVERGED;
        st->R = 0.0;
        st->omega = st->min_omega;
        if (!(bb == bb) || isinf(bb)) {
            st->done = 1;
            st->status = PF_NONFINITE;
        } else if (bb == 0.0) {
            st->done = 1;
            st->status = PF_OK;
        }
    }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_rho0(const double* partials, long long np, PcgState* st,
                                                          const double* dG) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (st->done) return;
    const double rz = sum_partials(partials, np, s_red);
    if (dG) defl_coef(partials, np, 1, dG, st, s_red);  // G^-1 W^T z
    if (threadIdx.x == 0) {
        st->rho_old = rz;
        if (!isfinite(rz)) {
            st->done = 1;
            st->status = PF_NONFINITE;
        }
    }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_alpha(const double* partials, long long np, PcgState* st) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (st->done) return;
    const double pq = sum_partials(partials, np, s_red);
    if (threadIdx.x == 0) {
        if (!isfinite(pq) || !isfinite(st->rho_old)) {
            st->done = 1;
            st->status = PF_NONFINITE;
        } else if (!(pq > 0.0)) {
            st->done = 1;
            st->status = PF_BREAKDOWN;
        } else {
            st->alpha = st->rho_old / pq;
        }
    }
}

// x += alpha p, r -= alpha q, partial sums of r.r; with rf (mixed form) also the FP32 copy
// of r that the V-cycle reads
__global__ void __launch_bounds__(kRedThreads) k_pcg_xr(long long n, const double* __restrict__ p,
                                                        const double* __restrict__ q, double* __restrict__ x,
                                                        double* __restrict__ r, const PcgState* st, double* partials,
                                                        float* __restrict__ rf) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (st->done) return;
    const double a = st->alpha;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] += a * p[i];
        const double ri = r[i] - a * q[i];
        r[i] = ri;
        if (rf) rf[i] = (float)ri;
        s += ri * ri;
    }
    s = block_sum<kRedThreads>(s, s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_check(const double* partials, long long np, PcgState* st) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (st->done) return;
    const double rr = sum_partials(partials, np, s_red);
    if (threadIdx.x == 0) {
        const double R = sqrt(rr) / st->norm_b;
        st->R = R;
        st->it += 1;
        if (!isfinite(R)) {
            st->done = 1;
            st->status = PF_NONFINITE;
        } else if (st->stop_le ? R <= st->tol : R < st->tol) {
            st->done = 1;
            st->status = PF_OK;
        } else if (st->it >= st->maxiter) {
            st->done = 1;
            st->status = PF_NOT_CONVERGED;
        } else {
            const double c = R < st->tol ? st->tol : (R > 0.1 ? 0.1 : R);
            st->omega = st->min_omega + st->d_omega / 2.0 * exp((-c + st->tol) * 500.0);
        }
    }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_beta(const double* partials, long long np, PcgState* st,
                                                          const double* dG) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (st->done) return;
    const double rz = sum_partials(partials, np, s_red);
    if (dG) defl_coef(partials, np, 1, dG, st, s_red);  // G^-1 W^T z
    if (threadIdx.x == 0) {
        if (!isfinite(rz)) {
            st->done = 1;
            st->status = PF_NONFINITE;
        } else {
            st->beta = rz / st->rho_old;
            st->rho_old = rz;
        }
    }
}

// component i % dof of a grid-stride loop, advanced without a 64-bit division per element
struct CompIter {
    int c, step, dof;
    __device__ CompIter(long long i0, long long stride, int d)
        : c((int)(i0 % d)), step((int)(stride % d)), dof(d) {}
    __device__ __forceinline__ void next() {
        c += step;
        if (c >= dof) c -= dof;
    }
};

// p = z + beta p (init: p = z); with the deflation field yf, z - Q coef in place of z
template <typename TZ>
__global__ void k_pcg_p(long long n, const TZ* __restrict__ z, double* __restrict__ p, const PcgState* st, int init,
                        const float* __restrict__ yf, int dof) {
    pdl_wait();
    pdl_trigger();
    if (st->done) return;
    const double b = st->beta;
    const double c0 = st->coef[0], c1 = st->coef[1], c2 = st->coef[2];
    const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    if (yf) {
        CompIter ci(i0, stride, dof);
#pragma unroll 4
        for (long long i = i0; i < n; i += stride, ci.next()) {
            const double zi = (double)z[i] - (double)yf[i] * (ci.c == 0 ? c0 : ci.c == 1 ? c1 : c2);
            p[i] = init ? zi : zi + b * p[i];
        }
    } else {
        for (long long i = i0; i < n; i += stride) {
            const double zi = (double)z[i];
            p[i] = init ? zi : zi + b * p[i];
        }
    }
}

__global__ void k_f2d(long long n, const float* __restrict__ a, double* __restrict__ b) {
    pdl_wait();
    pdl_trigger();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

// ---------------------------------------------------------------------------------------
// deflation (learned coarse-grid correction): PCG on the complement of span(Q) in the
// energy inner product (Saad, Yeung, Erhel, Guyomarc'h, SIAM J. Sci. Comput. 21 (2000)):
//   x0 = x + Q G^-1 Q^T (b - A x),  r0 = b - A x0,   G = Q^T A Q = Q^T W,
//   z = M r,  p = z - Q G^-1 W^T z (+ beta p),
// with the V-cycle M unchanged.  Q has three columns: the components of one nodal field
// (zero on constrained DOFs; DOF i is component i % dof, a third column is zero in 2D); G is
// inverted on the components whose diagonal is positive.
// ---------------------------------------------------------------------------------------
__global__ void k_defl_field(long long n, int dof, const double* __restrict__ y, const uint8_t* __restrict__ mask,
                             float* __restrict__ yf) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const bool con = mask && ((mask[i / dof] >> (int)(i % dof)) & 1);
        yf[i] = con ? 0.f : (float)y[i];
    }
}
__global__ void k_defl_comp(long long n, int dof, const float* __restrict__ yf, int c, double* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (int)(i % dof) == c ? (double)yf[i] : 0.0;
}
// partials of G_cd = q_c . W_d (9 per block, index c*3 + d, stride gridDim.x); Q is the
// FP32 field itself (an exact basis), W = K Q in FP64
__global__ void __launch_bounds__(kRedThreads) k_defl_gram(long long n, int dof, const float* __restrict__ yf,
                                                           const double* __restrict__ Wd, double* partials) {
    __shared__ double s_red[kRedThreads / 32];
    double g[9];
#pragma unroll
    for (int q = 0; q < 9; q++) g[q] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % dof);
        const double y = yf[i];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double t = y * Wd[d * n + i];
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
                if (cc == c) g[cc * 3 + d] += t;
        }
    }
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const double t = block_sum<kRedThreads>(g[q], s_red);
        if (threadIdx.x == 0) partials[(long long)q * gridDim.x + blockIdx.x] = t;
    }
}
// G^-1 over the components with a positive diagonal (the others get zero rows and columns)
__global__ void __launch_bounds__(kRedThreads) k_defl_ginv(const double* partials, long long np, double* dG) {
    __shared__ double s_red[kRedThreads / 32];
    double G[9];
    for (int q = 0; q < 9; q++) G[q] = sum_partials(partials + q * np, np, s_red);
    if (threadIdx.x != 0) return;
    // symmetrise, select the active components
    double A[3][3], I[3][3];
    int act[3];
    const double gmax = fmax(G[0], fmax(G[4], G[8]));
    for (int c = 0; c < 3; c++) act[c] = G[c * 4] > 1e-12 * gmax && gmax > 0.0;
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) {
            A[c][d] = (act[c] && act[d]) ? 0.5 * (G[c * 3 + d] + G[d * 3 + c]) : (c == d ? 1.0 : 0.0);
            I[c][d] = c == d ? 1.0 : 0.0;
        }
    // Gauss-Jordan on the SPD 3x3 (no pivoting needed)
    int ok = 1;
    for (int k = 0; k < 3; k++) {
        const double piv = A[k][k];
        if (!(piv > 0.0)) {
            ok = 0;
            break;
        }
        for (int j = 0; j < 3; j++) {
            A[k][j] /= piv;
            I[k][j] /= piv;
        }
        for (int i = 0; i < 3; i++)
            if (i != k) {
                const double f = A[i][k];
                for (int j = 0; j < 3; j++) {
                    A[i][j] -= f * A[k][j];
                    I[i][j] -= f * I[k][j];
                }
            }
    }
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) dG[c * 3 + d] = (ok && act[c] && act[d]) ? I[c][d] : 0.0;
}
// partials of s_c = q_c . r (3 per block)
__global__ void __launch_bounds__(kRedThreads) k_defl_qt(long long n, int dof, const double* __restrict__ r,
                                                         const float* __restrict__ yf, double* partials) {
    pdl_wait();  // r, and the partials the previous kernel reads
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    double a[3] = {0.0, 0.0, 0.0};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % dof);
        const double t = (double)yf[i] * r[i];
#pragma unroll
        for (int cc = 0; cc < 3; cc++)
            if (cc == c) a[cc] += t;
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const double t = block_sum<kRedThreads>(a[q], s_red);
        if (threadIdx.x == 0) partials[(long long)q * gridDim.x + blockIdx.x] = t;
    }
}
// st->coef = G^-1 (3 sums of partials starting at partials + off * np)
__device__ void defl_coef(const double* partials, long long np, int off, const double* dG, PcgState* st,
                          double* s_red) {
    double t[3];
    for (int q = 0; q < 3; q++) t[q] = sum_partials(partials + (off + q) * np, np, s_red);
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; c++) st->coef[c] = dG[c * 3] * t[0] + dG[c * 3 + 1] * t[1] + dG[c * 3 + 2] * t[2];
}
__global__ void __launch_bounds__(kRedThreads) k_defl_coef(const double* partials, long long np, const double* dG,
                                                           PcgState* st) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (st->done) return;
    defl_coef(partials, np, 0, dG, st, s_red);
}
// x += Q coef
__global__ void k_defl_xadd(long long n, int dof, const float* __restrict__ yf, double* __restrict__ x,
                            const PcgState* st) {
    pdl_wait();
    pdl_trigger();
    if (st->done) return;
    const double c0 = st->coef[0], c1 = st->coef[1], c2 = st->coef[2];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % dof);
        x[i] += (double)yf[i] * (c == 0 ? c0 : c == 1 ? c1 : c2);
    }
}
// partials of r.z (index 0) and t_d = W_d . z (indices 1..3)
template <typename TZ>
__global__ void __launch_bounds__(kRedThreads) k_dot_defl(long long n, const double* __restrict__ r,
                                                          const TZ* __restrict__ z, const double* __restrict__ Wd,
                                                          double* partials, const int* skip) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[kRedThreads / 32];
    if (skip && *skip) return;
    double a[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double zi = (double)z[i];
        a[0] += r[i] * zi;
        a[1] += Wd[i] * zi;
        a[2] += Wd[n + i] * zi;
        a[3] += Wd[2 * n + i] * zi;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double t = block_sum<kRedThreads>(a[q], s_red);
        if (threadIdx.x == 0) partials[(long long)q * gridDim.x + blockIdx.x] = t;
    }
}

static unsigned vec_blocks(long long n) {
    long long nb = (n + kRedThreads - 1) / kRedThreads;
    const long long cap = 8LL * kNumSM;
    if (nb > cap) nb = cap;
    if (nb < 1) nb = 1;
    return (unsigned)nb;
}

// ---------------------------------------------------------------------------------------
// level operators
// ---------------------------------------------------------------------------------------
// algorithmic bytes of one fine matvec launch: u, E, mask and out once each, plus the
// epilogue operands (b, dinv, xadd) and a dot operand other than u
template <typename T>
static double fine_mv_bytes(const pf_mg* mg, const T* u, const Epi<T>& e) {
    const Grid& g = mg->op->grid;
    const double D = (double)g.n_nodes * g.dof, tb = sizeof(T);
    const double te = sizeof(T) == 8 ? 8.0 : (mg->Eb ? 2.0 : 4.0);  // bytes per element scale
    double b = 2.0 * D * tb + (double)g.n_elem * te + (mg->mask ? (double)g.n_nodes : 0.0);
    if (e.mode == PF_EPI_RESID) b += D * tb;
    if (e.mode == PF_EPI_JACOBI) b += 2.0 * D * tb;
    if (e.mode == PF_EPI_JACOBI_ADD) b += 3.0 * D * tb;
    if (e.dot_partial && (const void*)e.dot_a != (const void*)u) b += D * tb;
    return b;
}

template <typename T>
static int fine_mv(pf_mg* mg, const T* u, const Epi<T>& epi, cudaStream_t st) {
    const bool rec = mg->profile && mg->pn < (int)mg->pev.size() / 2 &&
                     (mg->profile_which & (sizeof(T) == 8 ? 1 : 2)) != 0;
    if (rec) PF_CUDA(cudaEventRecord(mg->pev[2 * mg->pn], st));
    int s;
    if constexpr (sizeof(T) == 8)
        s = launch_fine_matvec<double, double>(mg->op, mg->E, u, mg->mask, epi, st);
    else if (mg->Eb)
        s = launch_fine_matvec<float, __nv_bfloat16>(mg->op, mg->Eb, u, mg->mask, epi, st);
    else
        s = launch_fine_matvec<float, float>(mg->op, mg->Ef, u, mg->mask, epi, st);
    if (s) return s;
    if (rec) {
        PF_CUDA(cudaEventRecord(mg->pev[2 * mg->pn + 1], st));
        mg->pbytes[mg->pn] = fine_mv_bytes<T>(mg, u, epi);
        mg->pn++;
    }
    return PF_OK;
}

template <typename T>
static int level_matvec(pf_mg* mg, int l, const T* u, const Epi<T>& epi, cudaStream_t st) {
    if (l == 0) return fine_mv<T>(mg, u, epi, st);
    if (l == 1 && mg->c1) return launch_coarse_matvec<T>(mg->c1, mg->L[1].g, u, epi, st);
    return launch_stencil_matvec<T>(mg->L[l].g, (const T*)mg->L[l].H, u, epi, st, true);
}

template <typename T>
static Epi<T> make_epi(int mode, const T* b, const T* x, const T* dinv, const T* xadd, T* out, const double* omega,
                       double scale, const int* skip) {
    Epi<T> e;
    e.mode = mode;
    e.b = b;
    e.x = x;
    e.dinv = dinv;
    e.xadd = xadd;
    e.out = out;
    e.omega = omega;
    e.omega_scale = scale;
    e.dot_partial = nullptr;
    e.dot_a = nullptr;
    e.dot_of_y = 0;
    e.skip = skip;
    return e;
}

// Approximate A_l x = b from x = 0; returns (through *res) the buffer holding x.
// b0 overrides the level-0 right-hand side.  dot: optional fused r.z partial at level 0.
template <typename T>
static int vcycle(pf_mg* mg, int l, const T* b0, T** res, double* dot_partials, const double* dot_a, cudaStream_t st,
                  bool x_ready = false) {
    Level& L = mg->L[l];
    const int* skip = &mg->st->done;
    const double* omega = &mg->st->omega;
    const T* b = (l == 0 && b0) ? b0 : (const T*)L.b;
    if (l == mg->nlev) {
        int s = dense_solve<T>(&mg->dense, b, (T*)L.x, skip, st);
        *res = (T*)L.x;
        return s;
    }
    const double scale = pow(mg->cfg.omega_boost, l);
    const T* dinv = (const T*)L.dinv;
    T* X = (T*)L.x;
    T* Tb = (T*)L.t;
    int s;
    if (!x_ready) {  // otherwise the restriction from the finer level did this sweep
        pf::count_launch();
        PF_CUDA(launch_pdl(k_jacobi0<T>, dim3(vec_blocks(L.ndof)), dim3(kRedThreads), 0, st, L.ndof, b, dinv, omega, scale, X, skip));
        PF_LAUNCH_CHECK("jacobi0 launch");
    }
    for (int k = 1; k < mg->cfg.n_smooth; k++) {
        if ((s = level_matvec<T>(mg, l, X, make_epi<T>(PF_EPI_JACOBI, b, X, dinv, nullptr, Tb, omega, scale, skip), st)))
            return s;
        T* tmp = X;
        X = Tb;
        Tb = tmp;
    }
    T* R = (T*)L.r;
    T* Eb = (T*)L.e;
    // the 'w' cycle repeats the coarse correction from the updated X at the levels of w_mask
    const int passes = (l < 32 && ((mg->cfg.w_mask >> l) & 1u)) ? 2 : 1;
    for (int pass = 0; pass < passes; pass++) {
        if ((s = level_matvec<T>(mg, l, X, make_epi<T>(PF_EPI_RESID, b, nullptr, nullptr, nullptr, R, omega, scale, skip), st)))
            return s;
        Jacobi0<T> j0;
        const bool fuse = l + 1 < mg->nlev;  // the coarsest level is solved directly
        if (fuse) {
            j0.x = (T*)mg->L[l + 1].x;
            j0.dinv = (const T*)mg->L[l + 1].dinv;
            j0.omega = omega;
            j0.scale = pow(mg->cfg.omega_boost, l + 1);
        }
        if ((s = launch_restrict<T, T>(L.g, R, (T*)mg->L[l + 1].b, skip, st, j0))) return s;
        T* ec;
        if ((s = vcycle<T>(mg, l + 1, nullptr, &ec, nullptr, nullptr, st, fuse))) return s;
        if ((s = launch_prolong<T>(L.g, ec, Eb, skip, st))) return s;
        for (int k = 0; k < mg->cfg.n_smooth; k++) {
            const bool last = k == mg->cfg.n_smooth - 1;
            if (!last) {
                if ((s = level_matvec<T>(mg, l, Eb, make_epi<T>(PF_EPI_JACOBI, R, Eb, dinv, nullptr, Tb, omega, scale, skip), st)))
                    return s;
                T* tmp = Eb;
                Eb = Tb;
                Tb = tmp;
            } else {
                Epi<T> ep = make_epi<T>(PF_EPI_JACOBI_ADD, R, Eb, dinv, X, X, omega, scale, skip);
                if (dot_partials && pass == passes - 1) {
                    ep.dot_partial = dot_partials;
                    if constexpr (sizeof(T) == 8) ep.dot_a = (const T*)dot_a;
                    ep.dot_of_y = 0;
                }
                if ((s = level_matvec<T>(mg, l, Eb, ep, st))) return s;
            }
        }
    }
    *res = X;
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// create / destroy
// ---------------------------------------------------------------------------------------
static void mg_free(pf_mg* mg) {
    for (int l = 0; l <= kMaxLevel; l++) {
        Level& L = mg->L[l];
        for (void* p : {L.b, L.x, L.t, L.r, L.e, L.dinv}) if (p) cudaFree(p);
        if (L.A64) cudaFree(L.A64);
        if (L.H) cudaFree(L.H);
        L = Level();
    }
    dense_free(&mg->dense);
    coarse_destroy(mg->c1);
    mg->c1 = nullptr;
    for (void* p : {(void*)mg->K0_dev, (void*)mg->Kc_dev, (void*)mg->elem_flag, (void*)mg->node_flag, (void*)mg->Ef,
                    (void*)mg->Eb, (void*)mg->yf, (void*)mg->Wd, (void*)mg->dG, (void*)mg->gscratch,
                    (void*)mg->r, (void*)mg->p, (void*)mg->q, (void*)mg->partials, (void*)mg->st,
                    (void*)mg->Eint, (void*)mg->bi, (void*)mg->xi})
        if (p) cudaFree(p);
    for (cudaGraphExec_t g : {mg->g_start[0], mg->g_start[1], mg->g_chunk})
        if (g) cudaGraphExecDestroy(g);
    if (mg->ev_in) cudaEventDestroy(mg->ev_in);
    if (mg->ev_out) cudaEventDestroy(mg->ev_out);
    if (mg->cs) cudaStreamDestroy(mg->cs);
    if (mg->h_snap) cudaFreeHost(mg->h_snap);
}

// the captured start and iteration graphs bake in pointers and the PCG variant
static void drop_graphs(pf_mg* mg) {
    for (cudaGraphExec_t& gx : mg->g_start)
        if (gx) cudaGraphExecDestroy(gx), gx = nullptr;
    if (mg->g_chunk) cudaGraphExecDestroy(mg->g_chunk), mg->g_chunk = nullptr;
}

static int dalloc(void** p, size_t bytes) {
    if (bytes == 0) bytes = 8;
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(PF_NO_MEMORY, "device allocation of %zu bytes failed", bytes);
    }
    return PF_OK;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_mg_create(const pf_op* op, const pf_mg_config* cfg, pf_mg** out) {
    if (!op || !cfg || !out) return fail(PF_BAD_ARG, "pf_mg_create: NULL argument");
    *out = nullptr;
    if (cfg->n_level < 1 || cfg->n_level > kMaxLevel) return fail(PF_BAD_ARG, "n_level must be in [1, %d]", kMaxLevel);
    if (cfg->n_smooth < 1 || cfg->n_smooth > 64) return fail(PF_BAD_ARG, "n_smooth must be in [1, 64]");
    if (cfg->precision < 0 || cfg->precision > 2)
        return fail(PF_BAD_ARG, "precision must be 0 (fp64), 1 (fp32 V-cycle) or 2 (fp32 V-cycle, bf16 densities)");
    const Grid& g = op->grid;
    // every level floors nel / 2 (core/CUDA/_mgm.py:24-27); the coarsest keeps an element per axis
    for (int a = 0; a < g.dim; a++)
        if ((g.nel[a] >> cfg->n_level) < 1)
            return fail(PF_BAD_ARG, "nel[%d]=%d has no element left after %d halvings", a, g.nel[a], cfg->n_level);
    pf_mg* mg = new pf_mg();
    mg->op = op;
    mg->cfg = *cfg;
    if (mg->cfg.check_every < 1) mg->cfg.check_every = 1;
    mg->fp32 = cfg->precision != 0 ? 1 : 0;
    mg->nlev = cfg->n_level;
    const size_t ts = mg->fp32 ? sizeof(float) : sizeof(double);
    int s = PF_OK;
    if (cfg->coarse_op != 0 && cfg->coarse_op != 1) {
        delete mg;
        return fail(PF_BAD_ARG, "coarse_op must be 0 (element operator on level 1 when available) or 1 (stencils)");
    }
    if (!(cfg->omega_fixed >= 0.0) || !(cfg->omega_fixed < 2.0)) {
        delete mg;
        return fail(PF_BAD_ARG, "omega_fixed must be 0 (the reference schedule) or a Jacobi weight in (0, 2)");
    }
    // level 1 element by element when it is smoothed (not the coarsest), its coarse elements
    // cover the fine grid (even element counts) and K0 allows it
    const bool even = g.nel[0] % 2 == 0 && g.nel[1] % 2 == 0 && (g.dim == 2 || g.nel[2] % 2 == 0);
    if (cfg->coarse_op == 0 && g.dim == 3 && mg->nlev >= 2 && even) {
        double coef[150];
        if (coarse_factorise(op, coef) == PF_OK) s = coarse_create(op, mg->fp32, &mg->c1);
        if (!s) set_error("");
    }
    Grid gl = g;
    for (int l = 0; l <= mg->nlev && !s; l++) {
        Level& L = mg->L[l];
        L.g = gl;
        L.ndof = gl.n_nodes * gl.dof;
        const size_t vb = (size_t)L.ndof * ts;
        if (l >= 1 || mg->fp32) s = s ? s : dalloc(&L.b, vb);
        s = s ? s : dalloc(&L.x, vb);
        if (l < mg->nlev) {
            s = s ? s : dalloc(&L.t, vb);
            s = s ? s : dalloc(&L.r, vb);
            s = s ? s : dalloc(&L.e, vb);
            s = s ? s : dalloc(&L.dinv, vb);
        }
        if (l >= 1) {
            const size_t nst = (size_t)gl.n_nodes * (gl.dim == 3 ? 27 : 9) * gl.dof * gl.dof;
            s = s ? s : dalloc((void**)&L.A64, nst * sizeof(double));
            if (l < mg->nlev && !(l == 1 && mg->c1)) s = s ? s : dalloc(&L.H, (size_t)stencil_half_size(gl) * ts);
        }
        gl = coarse_grid(gl);
    }
    long long gsc = 0;
    for (int l = 2; l <= mg->nlev; l++) {
        const long long need = galerkin_sep_scratch(mg->L[l - 1].g);
        if (need > gsc) gsc = need;
    }
    if (gsc > 0) s = s ? s : dalloc((void**)&mg->gscratch, (size_t)gsc * sizeof(double));
    const long long ncoarse = mg->L[mg->nlev].ndof;
    if (!s && ncoarse > 6144)
        s = fail(PF_BAD_ARG, "coarsest level has %lld DOF (> 6144): use more levels", ncoarse);
    if (!s) s = dense_alloc(&mg->dense, (int)ncoarse);
    const int nc = g.dim == 3 ? 8 : 4, nd = nc * g.dim;
    s = s ? s : dalloc((void**)&mg->K0_dev, nd * nd * sizeof(double));
    s = s ? s : dalloc((void**)&mg->Kc_dev, (size_t)nc * nd * nd * sizeof(double));
    const Grid g1 = coarse_grid(g);
    s = s ? s : dalloc((void**)&mg->elem_flag, (size_t)g1.n_elem);
    s = s ? s : dalloc((void**)&mg->node_flag, (size_t)g1.n_nodes);
    const long long n0 = mg->L[0].ndof;
    if (cfg->precision == 1) s = s ? s : dalloc((void**)&mg->Ef, (size_t)g.n_elem * sizeof(float));
    if (cfg->precision == 2) s = s ? s : dalloc((void**)&mg->Eb, (size_t)g.n_elem * sizeof(__nv_bfloat16));
    s = s ? s : dalloc((void**)&mg->r, n0 * sizeof(double));
    s = s ? s : dalloc((void**)&mg->p, n0 * sizeof(double));
    s = s ? s : dalloc((void**)&mg->q, n0 * sizeof(double));
    // partial sums of the FP64 PCG matvec and (mixed form) of the FP32 V-cycle matvec
    long long np = fine_matvec_num_blocks(op, 0);
    if (mg->fp32 && fine_matvec_num_blocks(op, 1) > np) np = fine_matvec_num_blocks(op, 1);
    if (np < 8 * kNumSM) np = 8 * kNumSM;
    for (int l = 1; l < mg->nlev; l++) np = np > stencil_matvec_num_blocks(mg->L[l].g) ? np : stencil_matvec_num_blocks(mg->L[l].g);
    if (np < 9LL * 8 * kNumSM) np = 9LL * 8 * kNumSM;  // the deflation's 9 sums per reduction block
    mg->npartials = np;
    s = s ? s : dalloc((void**)&mg->partials, np * sizeof(double));
    s = s ? s : dalloc((void**)&mg->st, sizeof(PcgState));
    s = s ? s : dalloc((void**)&mg->Eint, (size_t)g.n_elem * sizeof(double));
    s = s ? s : dalloc((void**)&mg->bi, n0 * sizeof(double));
    s = s ? s : dalloc((void**)&mg->xi, n0 * sizeof(double));
    if (!s && (cudaStreamCreateWithFlags(&mg->cs, cudaStreamNonBlocking) != cudaSuccess ||
               cudaEventCreateWithFlags(&mg->ev_in, cudaEventDisableTiming) != cudaSuccess ||
               cudaEventCreateWithFlags(&mg->ev_out, cudaEventDisableTiming) != cudaSuccess))
        s = fail(PF_CUDA_ERROR, "stream / event creation failed");
    if (!s && cudaMallocHost((void**)&mg->h_snap, 2 * sizeof(PcgState)) != cudaSuccess)
        s = fail(PF_NO_MEMORY, "pinned allocation failed");
    if (!s) {
        std::vector<double> Kc((size_t)nc * nd * nd);
        galerkin_child_matrices(g.dim, op->K0, Kc.data());
        if (cudaMemcpy(mg->K0_dev, op->K0, nd * nd * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(mg->Kc_dev, Kc.data(), Kc.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            s = fail(PF_CUDA_ERROR, "upload of element matrices failed");
    }
    for (int i = 0; i < 6 && !s; i++)
        if (cudaEventCreate(&mg->ev[i]) != cudaSuccess) s = fail(PF_CUDA_ERROR, "event creation failed");
    if (s) {
        mg_free(mg);
        delete mg;
        return s;
    }
    *out = mg;
    return PF_OK;
}

extern "C" int pf_mg_destroy(pf_mg* mg) {
    if (!mg) return PF_OK;
    cudaDeviceSynchronize();
    for (int i = 0; i < 6; i++)
        if (mg->ev[i]) cudaEventDestroy(mg->ev[i]);
    for (cudaEvent_t e : mg->pev) cudaEventDestroy(e);
    mg_free(mg);
    delete mg;
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// setup
// ---------------------------------------------------------------------------------------
extern "C" int pf_mg_setup(pf_mg* mg, const double* E, const uint8_t* node_mask, void* stream) {
    if (!mg || !E) return fail(PF_BAD_ARG, "pf_mg_setup: NULL argument");
    cudaStream_t st = as_stream(stream);
    PF_CUDA(cudaEventRecord(mg->ev[0], st));
    PF_CUDA(cudaMemcpyAsync(mg->Eint, E, sizeof(double) * mg->op->grid.n_elem, cudaMemcpyDeviceToDevice, st));
    E = mg->Eint;
    mg->E = E;
    if (node_mask != mg->g_mask) drop_graphs(mg);  // graphs bake the mask pointer in: recapture
    if (mg->defl) {  // A Q changes with the densities: the deflation space is set again after setup
        mg->defl = 0;
        drop_graphs(mg);
    }
    mg->mask = node_mask;
    mg->ready = false;
    int s;
    Level& L0 = mg->L[0];
    const Grid& g = mg->op->grid;
    // level 0: inverse diagonal
    if (mg->fp32) {
        if ((s = launch_diagonal<float>(mg->op, E, node_mask, (float*)L0.dinv, st))) return s;
        pf::count_launch();
        k_recip<float><<<vec_blocks(L0.ndof), kRedThreads, 0, st>>>(L0.ndof, (float*)L0.dinv);
        if (mg->Eb) {
            if ((s = launch_d2bf(g.n_elem, E, mg->Eb, st))) return s;
        } else if ((s = launch_d2f(g.n_elem, E, mg->Ef, st))) {
            return s;
        }
    } else {
        if ((s = launch_diagonal<double>(mg->op, E, node_mask, (double*)L0.dinv, st))) return s;
        pf::count_launch();
        k_recip<double><<<vec_blocks(L0.ndof), kRedThreads, 0, st>>>(L0.ndof, (double*)L0.dinv);
    }
    PF_LAUNCH_CHECK("recip launch");
    // level 1
    const Grid g1 = coarse_grid(g);
    if (node_mask) {
        if ((s = launch_coarse_flags(g, node_mask, mg->elem_flag, mg->node_flag, st))) return s;
    } else {
        PF_CUDA(cudaMemsetAsync(mg->elem_flag, 0, (size_t)g1.n_elem, st));
        PF_CUDA(cudaMemsetAsync(mg->node_flag, 0, (size_t)g1.n_nodes, st));
    }
    if ((s = launch_galerkin_l0(g, E, node_mask, mg->elem_flag, mg->node_flag, mg->K0_dev, mg->Kc_dev, mg->L[1].A64, st)))
        return s;
    for (int l = 2; l <= mg->nlev; l++)
        if ((s = launch_galerkin_sep(mg->L[l - 1].g, mg->L[l - 1].A64, mg->L[l].A64, mg->gscratch, st))) return s;
    for (int l = 1; l < mg->nlev; l++) {
        Level& L = mg->L[l];
        const bool half = L.H != nullptr;  // level 1 with the element operator has no stencil copy
        if (mg->fp32) {
            if ((s = launch_stencil_dinv<float>(L.g, L.A64, (float*)L.dinv, st))) return s;
            if (half && (s = launch_stencil_half<float>(L.g, L.A64, (float*)L.H, st))) return s;
        } else {
            if ((s = launch_stencil_dinv<double>(L.g, L.A64, (double*)L.dinv, st))) return s;
            if (half && (s = launch_stencil_half<double>(L.g, L.A64, (double*)L.H, st))) return s;
        }
    }
    if (mg->c1) {
        bool moved = false;
        if ((s = coarse_setup(mg->c1, E, node_mask, mg->elem_flag, mg->node_flag, mg->K0_dev, st, &moved))) return s;
        if (moved) drop_graphs(mg);  // the captured graphs hold the old dirty storage: recapture
    }
    // coarsest: dense factor and inverse
    Dense& D = mg->dense;
    PF_CUDA(cudaMemsetAsync(D.M, 0, (size_t)D.np * D.np * sizeof(double), st));
    if ((s = launch_stencil_to_dense(mg->L[mg->nlev].g, mg->L[mg->nlev].A64, D.M, D.np, st))) return s;
    if ((s = dense_factor_invert(&D, mg->cfg.coarse_beta, st))) return s;
    PF_CUDA(cudaEventRecord(mg->ev[1], st));
    mg->ready = true;
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// V-cycle (public) and PCG
// ---------------------------------------------------------------------------------------
__global__ void k_init_state(PcgState* st, double tol, int maxiter, double min_omega, double d_omega, double omega,
                             int stop_le) {
    pdl_wait();
    pdl_trigger();
    PcgState h;
    memset(&h, 0, sizeof(h));
    h.tol = tol;
    h.maxiter = maxiter;
    h.min_omega = min_omega;
    h.d_omega = d_omega;
    h.omega = omega;
    h.status = PF_NOT_CONVERGED;
    h.stop_le = stop_le;
    *st = h;
}

static int init_state(pf_mg* mg, double tol, int maxiter, double omega, cudaStream_t st) {
    // the schedule's floor and span; a fixed weight is a floor with no span
    const bool fixed = mg->cfg.omega_fixed > 0.0;
    const double min_omega = fixed ? mg->cfg.omega_fixed : fmax(mg->cfg.omega / 2.0, mg->cfg.min_omega);
    const double d_omega = fixed ? 0.0 : mg->cfg.omega - min_omega;
    pf::count_launch();
    PF_CUDA(launch_pdl(k_init_state, dim3(1), dim3(1), 0, st, mg->st, tol, maxiter, min_omega, d_omega, omega, 0));
    PF_LAUNCH_CHECK("state init");
    return PF_OK;
}

extern "C" int pf_mg_vcycle(pf_mg* mg, const double* r, double* z, double omega, void* stream) {
    if (!mg || !r || !z) return fail(PF_BAD_ARG, "pf_mg_vcycle: NULL argument");
    if (!mg->ready) return fail(PF_BAD_ARG, "pf_mg_vcycle: call pf_mg_setup first");
    cudaStream_t st = as_stream(stream);
    int s;
    if ((s = init_state(mg, 0.0, 1, omega, st))) return s;
    const long long n = mg->L[0].ndof;
    if (mg->fp32) {
        pf::count_launch();
        PF_CUDA(launch_pdl(k_d2f_skip, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, r, (float*)mg->L[0].b, nullptr));
        float* res;
        if ((s = vcycle<float>(mg, 0, (const float*)mg->L[0].b, &res, nullptr, nullptr, st))) return s;
        pf::count_launch();
        PF_CUDA(launch_pdl(k_f2d, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, res, z));
    } else {
        double* res;
        if ((s = vcycle<double>(mg, 0, r, &res, nullptr, nullptr, st))) return s;
        PF_CUDA(cudaMemcpyAsync(z, res, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    PF_LAUNCH_CHECK("vcycle");
    return PF_OK;
}

// apply the preconditioner to mg->r, leave r.z partials in mg->partials and return z
// (mixed form: r32_ready = the FP32 copy of r is already in the V-cycle's input)
static int precondition(pf_mg* mg, const void** z_out, long long* np_out, cudaStream_t st, bool r32_ready) {
    const long long n = mg->L[0].ndof;
    int s;
    if (mg->fp32) {
        if (!r32_ready) {
            pf::count_launch();
            PF_CUDA(launch_pdl(k_d2f_skip, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, mg->r, (float*)mg->L[0].b,
                               &mg->st->done));
        }
        float* res;
        if ((s = vcycle<float>(mg, 0, (const float*)mg->L[0].b, &res, nullptr, nullptr, st))) return s;
        pf::count_launch();
        if (mg->defl)  // r.z and W^T z
            PF_CUDA(launch_pdl(k_dot_defl<float>, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, (const double*)mg->r,
                               (const float*)res, (const double*)mg->Wd, mg->partials, (const int*)&mg->st->done));
        else
            PF_CUDA(launch_pdl(k_dot_partial<float>, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, mg->r, res, mg->partials, &mg->st->done));
        PF_LAUNCH_CHECK("dot launch");
        *z_out = res;
        *np_out = vec_blocks(n);
    } else {
        double* res;
        if (mg->defl) {
            if ((s = vcycle<double>(mg, 0, mg->r, &res, nullptr, nullptr, st))) return s;
            pf::count_launch();
            PF_CUDA(launch_pdl(k_dot_defl<double>, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, (const double*)mg->r,
                               (const double*)res, (const double*)mg->Wd, mg->partials, (const int*)&mg->st->done));
            PF_LAUNCH_CHECK("dot launch");
            *np_out = vec_blocks(n);
        } else {
            if ((s = vcycle<double>(mg, 0, mg->r, &res, mg->partials, mg->r, st))) return s;
            *np_out = fine_matvec_num_blocks(mg->op, 0);
        }
        *z_out = res;
    }
    return PF_OK;
}

static int update_p(pf_mg* mg, const void* z, int init, cudaStream_t st) {
    const long long n = mg->L[0].ndof;
    pf::count_launch();
    if (mg->fp32)
        PF_CUDA(launch_pdl(k_pcg_p<float>, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, (const float*)z, mg->p, mg->st, init,
                           (const float*)(mg->defl ? mg->yf : nullptr), mg->op->grid.dof));
    else
        PF_CUDA(launch_pdl(k_pcg_p<double>, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, (const double*)z, mg->p, mg->st, init,
                           (const float*)(mg->defl ? mg->yf : nullptr), mg->op->grid.dof));
    PF_LAUNCH_CHECK("p update launch");
    return PF_OK;
}

static int pcg_iteration(pf_mg* mg, double* x, cudaStream_t st) {
    const long long n = mg->L[0].ndof;
    const int* skip = &mg->st->done;
    int s;
    // q = K p, p.q
    Epi<double> e = make_epi<double>(PF_EPI_STORE, nullptr, nullptr, nullptr, nullptr, mg->q, nullptr, 1.0, skip);
    e.dot_partial = mg->partials;
    e.dot_a = mg->p;
    e.dot_of_y = 1;
    if ((s = fine_mv<double>(mg, mg->p, e, st))) return s;
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_alpha, dim3(1), dim3(kRedThreads), 0, st, mg->partials, fine_matvec_num_blocks(mg->op, 0), mg->st));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_xr, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, mg->p, mg->q, x, mg->r, mg->st, mg->partials,
                       mg->fp32 ? (float*)mg->L[0].b : (float*)nullptr));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_check, dim3(1), dim3(kRedThreads), 0, st, mg->partials, vec_blocks(n), mg->st));
    PF_LAUNCH_CHECK("pcg launch");
    const void* z;
    long long np;
    if ((s = precondition(mg, &z, &np, st, true))) return s;
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_beta, dim3(1), dim3(kRedThreads), 0, st, mg->partials, np, mg->st,
                       (const double*)(mg->defl ? mg->dG : nullptr)));
    PF_LAUNCH_CHECK("beta launch");
    return update_p(mg, z, 0, st);
}

// Capture the launches `body` issues on the private stream into an executable graph.
template <typename F>
static int capture(pf_mg* mg, F body, cudaGraphExec_t* out, unsigned long long* nodes) {
    const unsigned long long c0 = launch_count();
    PF_CUDA(cudaStreamBeginCapture(mg->cs, cudaStreamCaptureModeThreadLocal));
    int s = body(mg->cs);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(mg->cs, &graph);
    *nodes = launch_count() - c0;
    uncount_launch(*nodes);  // captured, not launched
    if (s) {
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    if (e != cudaSuccess) return check_cuda(e, "stream capture");
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return check_cuda(e, "graph instantiate");
    return PF_OK;
}

// r = b - K x (or b with x = 0), ||b||, z = M r, p = z, rho = r.z
static int solve_start(pf_mg* mg, int use_x0, cudaStream_t st) {
    const long long n = mg->L[0].ndof;
    int s;
    if (use_x0) {
        Epi<double> e = make_epi<double>(PF_EPI_RESID, mg->bi, nullptr, nullptr, nullptr, mg->r, nullptr, 1.0, nullptr);
        if ((s = fine_mv<double>(mg, mg->xi, e, st))) return s;
    } else {
        PF_CUDA(cudaMemsetAsync(mg->xi, 0, n * sizeof(double), st));
        PF_CUDA(cudaMemcpyAsync(mg->r, mg->bi, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    pf::count_launch();
    PF_CUDA(launch_pdl(k_dot_partial<double>, dim3(vec_blocks(n)), dim3(kRedThreads), 0, st, n, mg->bi, mg->bi, mg->partials, nullptr));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_normb, dim3(1), dim3(kRedThreads), 0, st, mg->partials, vec_blocks(n), mg->st));
    PF_LAUNCH_CHECK("pcg start");
    if (mg->defl) {  // x += Q G^-1 Q^T r, r = b - A x
        const unsigned vb = vec_blocks(n);
        pf::count_launch(3);
        PF_CUDA(launch_pdl(k_defl_qt, dim3(vb), dim3(kRedThreads), 0, st, n, mg->op->grid.dof, (const double*)mg->r,
                           (const float*)mg->yf, mg->partials));
        PF_CUDA(launch_pdl(k_defl_coef, dim3(1), dim3(kRedThreads), 0, st, (const double*)mg->partials, (long long)vb,
                           (const double*)mg->dG, mg->st));
        PF_CUDA(launch_pdl(k_defl_xadd, dim3(vb), dim3(kRedThreads), 0, st, n, mg->op->grid.dof, (const float*)mg->yf,
                           mg->xi, (const PcgState*)mg->st));
        PF_LAUNCH_CHECK("deflated start");
        Epi<double> e = make_epi<double>(PF_EPI_RESID, mg->bi, nullptr, nullptr, nullptr, mg->r, nullptr, 1.0, nullptr);
        if ((s = fine_mv<double>(mg, mg->xi, e, st))) return s;
    }
    const void* z;
    long long np;
    if ((s = precondition(mg, &z, &np, st, false))) return s;
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_rho0, dim3(1), dim3(kRedThreads), 0, st, mg->partials, np, mg->st,
                       (const double*)(mg->defl ? mg->dG : nullptr)));
    return update_p(mg, z, 1, st);
}

extern "C" int pf_mg_solve(pf_mg* mg, const double* b, double* x, int use_x0, double tol, int maxiter,
                           pf_solve_info* info, void* stream) {
    if (!mg || !b || !x) return fail(PF_BAD_ARG, "pf_mg_solve: NULL argument");
    if (!mg->ready) return fail(PF_BAD_ARG, "pf_mg_solve: call pf_mg_setup first");
    if (maxiter < 0) return fail(PF_BAD_ARG, "maxiter must be >= 0");
    cudaStream_t us = as_stream(stream), cs = mg->cs;
    const long long n = mg->L[0].ndof;
    const int C = mg->cfg.check_every;
    const bool graphs = !mg->profile;
    int s;
    // the private stream starts after everything already queued on the caller's stream
    PF_CUDA(cudaEventRecord(mg->ev_in, us));
    PF_CUDA(cudaStreamWaitEvent(cs, mg->ev_in, 0));
    if ((s = init_state(mg, tol, maxiter, 0.0, cs))) return s;
    mg->pn = 0;
    PF_CUDA(cudaEventRecord(mg->ev[2], cs));
    PF_CUDA(cudaMemcpyAsync(mg->bi, b, n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    if (use_x0) PF_CUDA(cudaMemcpyAsync(mg->xi, x, n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    const int v = use_x0 ? 1 : 0;
    if (graphs) {
        if (!mg->g_start[v] &&
            (s = capture(mg, [&](cudaStream_t c) { return solve_start(mg, use_x0, c); }, &mg->g_start[v],
                         &mg->g_start_nodes[v])))
            return s;
        PF_CUDA(cudaGraphLaunch(mg->g_start[v], cs));
        count_launch(mg->g_start_nodes[v]);
    } else if ((s = solve_start(mg, use_x0, cs))) {
        return s;
    }
    if (graphs && !mg->g_chunk && maxiter > 0) {
        auto body = [&](cudaStream_t c) {
            for (int k = 0; k < C; k++) {
                int r = pcg_iteration(mg, mg->xi, c);
                if (r) return r;
            }
            return (int)PF_OK;
        };
        if ((s = capture(mg, body, &mg->g_chunk, &mg->g_chunk_nodes))) return s;
    }
    mg->g_mask = mg->mask;
    // iterate in chunks of C, polling the completion flag of the previous chunk while the
    // next one is queued; iterations past convergence or maxiter are no-ops on the device
    int queued = 0, chunk = 0;
    while (queued < maxiter) {
        if (graphs) {
            PF_CUDA(cudaGraphLaunch(mg->g_chunk, cs));
            count_launch(mg->g_chunk_nodes);
        } else {
            for (int k = 0; k < C; k++)
                if ((s = pcg_iteration(mg, mg->xi, cs))) return s;
        }
        queued += C;
        const int slot = chunk & 1;
        PF_CUDA(cudaMemcpyAsync(&mg->h_snap[slot], mg->st, sizeof(PcgState), cudaMemcpyDeviceToHost, cs));
        PF_CUDA(cudaEventRecord(mg->ev[3 + slot], cs));
        if (chunk > 0) {
            const int prev = slot ^ 1;
            PF_CUDA(cudaEventSynchronize(mg->ev[3 + prev]));
            if (mg->h_snap[prev].done) break;
        }
        chunk++;
    }
    PF_CUDA(cudaMemcpyAsync(x, mg->xi, n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    PF_CUDA(cudaEventRecord(mg->ev[5], cs));
    PF_CUDA(cudaEventRecord(mg->ev_out, cs));
    PF_CUDA(cudaStreamWaitEvent(us, mg->ev_out, 0));
    PF_CUDA(cudaStreamSynchronize(cs));
    PcgState fin;
    PF_CUDA(cudaMemcpy(&fin, mg->st, sizeof(PcgState), cudaMemcpyDeviceToHost));
    float setup_ms = 0.f, solve_ms = 0.f;
    if (cudaEventElapsedTime(&setup_ms, mg->ev[0], mg->ev[1]) != cudaSuccess) setup_ms = 0.f;
    if (cudaEventElapsedTime(&solve_ms, mg->ev[2], mg->ev[5]) != cudaSuccess) solve_ms = 0.f;
    cudaGetLastError();
    if (info) {
        info->iterations = fin.it;
        info->status = fin.done ? fin.status : PF_NOT_CONVERGED;
        info->residual = fin.R;
        info->setup_ms = setup_ms;
        info->solve_ms = solve_ms;
    }
    if (mg->profile) {
        mg->prof_ms = 0.0;
        mg->prof_bytes = 0.0;
        mg->prof_launches = mg->pn;
        for (int i = 0; i < mg->pn; i++) {
            float ms = 0.f;
            PF_CUDA(cudaEventElapsedTime(&ms, mg->pev[2 * i], mg->pev[2 * i + 1]));
            mg->prof_ms += ms;
            mg->prof_bytes += mg->pbytes[i];
        }
    }
    int fpiv = 0;
    PF_CUDA(cudaMemcpy(&fpiv, mg->dense.fail, sizeof(int), cudaMemcpyDeviceToHost));
    if (fpiv) {
        if (info) info->status = PF_FACTOR_FAILED;
        return fail(PF_FACTOR_FAILED, "coarse Cholesky: non-positive pivot at row %d", fpiv - 1);
    }
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// plain CG (identity preconditioner): workspace = r | p | q | partials | state
// ---------------------------------------------------------------------------------------
static long long cg_npartials(const pf_op* op) {
    long long np = fine_matvec_num_blocks(op, 0);
    return np > 8LL * kNumSM ? np : 8LL * kNumSM;
}

extern "C" size_t pf_cg_workspace_size(const pf_op* op) {
    if (!op) return 0;
    const long long n = op->grid.n_nodes * op->grid.dof;
    return (size_t)(3 * n + cg_npartials(op) + (sizeof(PcgState) + 7) / 8 + 1);
}

extern "C" int pf_cg_solve(const pf_op* op, const double* E, const uint8_t* node_mask, const double* b, double* x,
                           int use_x0, double tol, int maxiter, double* work, pf_solve_info* info, void* stream) {
    if (!op || !E || !b || !x || !work) return fail(PF_BAD_ARG, "pf_cg_solve: NULL argument");
    if (maxiter < 0) return fail(PF_BAD_ARG, "maxiter must be >= 0");
    cudaStream_t st = as_stream(stream);
    const long long n = op->grid.n_nodes * op->grid.dof, npart = cg_npartials(op);
    double *r = work, *p = work + n, *q = work + 2 * n, *partials = work + 3 * n;
    PcgState* S = (PcgState*)(partials + npart);
    const int* skip = &S->done;
    pf::count_launch();
    // cupyx cg (the reference CG solver, solvers/CUDA/_solvers.py:114-127) stops at ||r|| <= tol ||b||
    PF_CUDA(launch_pdl(k_init_state, dim3(1), dim3(1), 0, st, S, tol, maxiter, 0.0, 0.0, 0.0, 1));
    if (use_x0) {
        Epi<double> e = make_epi<double>(PF_EPI_RESID, b, nullptr, nullptr, nullptr, r, nullptr, 1.0, nullptr);
        int s = launch_fine_matvec<double, double>(op, E, x, node_mask, e, st);
        if (s) return s;
    } else {
        PF_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), st));
        PF_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    const unsigned vb = vec_blocks(n);
    pf::count_launch();
    PF_CUDA(launch_pdl(k_dot_partial<double>, dim3(vb), dim3(kRedThreads), 0, st, n, b, b, partials, nullptr));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_normb, dim3(1), dim3(kRedThreads), 0, st, partials, vb, S));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_dot_partial<double>, dim3(vb), dim3(kRedThreads), 0, st, n, r, r, partials, skip));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_rho0, dim3(1), dim3(kRedThreads), 0, st, partials, vb, S, (const double*)nullptr));
    pf::count_launch();
    PF_CUDA(launch_pdl(k_pcg_p<double>, dim3(vb), dim3(kRedThreads), 0, st, n, r, p, S, 1, (const float*)nullptr, 3));
    PF_LAUNCH_CHECK("cg start");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    PcgState h;
    int it = 0;
    const long long nbm = fine_matvec_num_blocks(op, 0);
    while (it < maxiter) {
        const int chunk = (maxiter - it) < 8 ? (maxiter - it) : 8;
        for (int k = 0; k < chunk; k++) {
            Epi<double> e = make_epi<double>(PF_EPI_STORE, nullptr, nullptr, nullptr, nullptr, q, nullptr, 1.0, skip);
            e.dot_partial = partials;
            e.dot_a = p;
            e.dot_of_y = 1;
            int s = launch_fine_matvec<double, double>(op, E, p, node_mask, e, st);
            if (s) return s;
            pf::count_launch();
            PF_CUDA(launch_pdl(k_pcg_alpha, dim3(1), dim3(kRedThreads), 0, st, partials, nbm, S));
            pf::count_launch();
            PF_CUDA(launch_pdl(k_pcg_xr, dim3(vb), dim3(kRedThreads), 0, st, n, p, q, x, r, S, partials, (float*)nullptr));
            pf::count_launch();
            PF_CUDA(launch_pdl(k_pcg_check, dim3(1), dim3(kRedThreads), 0, st, partials, vb, S));
            pf::count_launch();
            PF_CUDA(launch_pdl(k_pcg_beta, dim3(1), dim3(kRedThreads), 0, st, partials, vb, S, (const double*)nullptr));
            pf::count_launch();
            PF_CUDA(launch_pdl(k_pcg_p<double>, dim3(vb), dim3(kRedThreads), 0, st, n, r, p, S, 0, (const float*)nullptr, 3));
        }
        PF_LAUNCH_CHECK("cg iteration");
        it += chunk;
        PF_CUDA(cudaMemcpyAsync(&h, S, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaStreamSynchronize(st));
        if (h.done) break;
    }
    cudaEventRecord(e1, st);
    PF_CUDA(cudaMemcpyAsync(&h, S, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
    PF_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (info) {
        info->iterations = h.it;
        info->status = h.done ? h.status : PF_NOT_CONVERGED;
        info->residual = h.R;
        info->setup_ms = 0.0;
        info->solve_ms = ms;
    }
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// deflation space: Q = the three components of a nodal field, W = A Q, G^-1 = (Q^T W)^-1
// ---------------------------------------------------------------------------------------
extern "C" int pf_mg_set_deflation(pf_mg* mg, const double* y, void* stream) {
    if (!mg) return fail(PF_BAD_ARG, "pf_mg_set_deflation: NULL solver");
    if (!y) {
        if (mg->defl) drop_graphs(mg);  // the captured iterations are the deflated ones
        mg->defl = 0;
        return PF_OK;
    }
    if (!mg->ready) return fail(PF_BAD_ARG, "pf_mg_set_deflation: call pf_mg_setup first");
    cudaStream_t st = as_stream(stream);
    const long long n = mg->L[0].ndof;
    int s = PF_OK;
    if (!mg->yf) {
        s = dalloc((void**)&mg->yf, (size_t)n * sizeof(float));
        s = s ? s : dalloc((void**)&mg->Wd, (size_t)3 * n * sizeof(double));
        s = s ? s : dalloc((void**)&mg->dG, 16 * sizeof(double));
        if (s) return s;
    }
    const unsigned vb = vec_blocks(n);
    pf::count_launch();
    const int dof = mg->op->grid.dof;
    k_defl_field<<<vb, kRedThreads, 0, st>>>(n, dof, y, mg->mask, mg->yf);
    PF_LAUNCH_CHECK("deflation field launch");
    if (dof == 2) PF_CUDA(cudaMemsetAsync(mg->Wd + 2 * n, 0, (size_t)n * sizeof(double), st));
    // W_c = A q_c through the FP64 fine matvec (q as scratch), kept in FP64: with W rounded to
    // FP32 the projection leaves Q^T r a drift of the rounding error every iteration, nothing
    // in the deflated iteration removes it, and the solve diverges
    for (int c = 0; c < dof; c++) {
        pf::count_launch();
        k_defl_comp<<<vb, kRedThreads, 0, st>>>(n, dof, mg->yf, c, mg->q);
        PF_LAUNCH_CHECK("deflation column launch");
        Epi<double> e = make_epi<double>(PF_EPI_STORE, nullptr, nullptr, nullptr, nullptr, mg->Wd + (size_t)c * n,
                                         nullptr, 1.0, nullptr);
        if ((s = launch_fine_matvec<double, double>(mg->op, mg->E, mg->q, mg->mask, e, st))) return s;
    }
    pf::count_launch(2);
    k_defl_gram<<<vb, kRedThreads, 0, st>>>(n, dof, mg->yf, (const double*)mg->Wd, mg->partials);
    k_defl_ginv<<<1, kRedThreads, 0, st>>>(mg->partials, (long long)vb, mg->dG);
    PF_LAUNCH_CHECK("deflation Gram launch");
    if (!mg->defl) drop_graphs(mg);  // the captured iterations are the plain ones
    mg->defl = 1;
    return PF_OK;
}

extern "C" int pf_mg_level_matvec(pf_mg* mg, int level, const void* u, void* y, void* stream) {
    if (!mg || !u || !y) return fail(PF_BAD_ARG, "pf_mg_level_matvec: NULL argument");
    if (!mg->ready) return fail(PF_BAD_ARG, "pf_mg_level_matvec: call pf_mg_setup first");
    if (level < 0 || level >= mg->nlev)
        return fail(PF_BAD_ARG, "pf_mg_level_matvec: level must be in [0, %d)", mg->nlev);
    if (u == y) return fail(PF_BAD_ARG, "pf_mg_level_matvec: u and y must not alias");
    cudaStream_t st = as_stream(stream);
    if (mg->fp32) {
        Epi<float> e = make_epi<float>(PF_EPI_STORE, nullptr, nullptr, nullptr, nullptr, (float*)y, nullptr, 1.0, nullptr);
        return level_matvec<float>(mg, level, (const float*)u, e, st);
    }
    Epi<double> e = make_epi<double>(PF_EPI_STORE, nullptr, nullptr, nullptr, nullptr, (double*)y, nullptr, 1.0, nullptr);
    return level_matvec<double>(mg, level, (const double*)u, e, st);
}

extern "C" int pf_mg_level_info(const pf_mg* mg, int* h_elem_level1, int* h_dirty) {
    if (!mg || !h_elem_level1 || !h_dirty) return fail(PF_BAD_ARG, "pf_mg_level_info: NULL argument");
    *h_elem_level1 = mg->c1 ? 1 : 0;
    *h_dirty = mg->c1 ? mg->c1->ndirty : 0;
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// profiling of the fine-level matvec inside a solve
// ---------------------------------------------------------------------------------------
extern "C" int pf_mg_set_profiling(pf_mg* mg, int max_launches) {
    if (!mg || max_launches < 0) return fail(PF_BAD_ARG, "pf_mg_set_profiling: bad argument");
    PF_CUDA(cudaDeviceSynchronize());
    for (cudaEvent_t e : mg->pev) cudaEventDestroy(e);
    mg->pev.clear();
    mg->pbytes.clear();
    mg->profile = max_launches > 0;
    mg->pn = 0;
    for (int i = 0; i < 2 * max_launches; i++) {
        cudaEvent_t e;
        PF_CUDA(cudaEventCreate(&e));
        mg->pev.push_back(e);
    }
    mg->pbytes.assign(max_launches, 0.0);
    return PF_OK;
}

extern "C" int pf_mg_profile_select(pf_mg* mg, int which) {
    if (!mg || which < 1 || which > 3) return fail(PF_BAD_ARG, "pf_mg_profile_select: which must be 1, 2 or 3");
    mg->profile_which = which;
    return PF_OK;
}

extern "C" int pf_mg_profile(const pf_mg* mg, double* h_ms, long long* h_launches, double* h_bytes) {
    if (!mg || !h_ms || !h_launches || !h_bytes) return fail(PF_BAD_ARG, "pf_mg_profile: NULL argument");
    *h_ms = mg->prof_ms;
    *h_launches = mg->prof_launches;
    *h_bytes = mg->prof_bytes;
    return PF_OK;
}
