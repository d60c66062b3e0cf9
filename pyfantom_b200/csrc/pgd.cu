// Projected gradient descent (pyFANTOM/Optimizers/CUDA/PGD.py:6-372): the vector work of
// one iteration.
//
//   stats     one pass over (x, df, x_last, df_last) for the scalars of the step-size rule
//             (PGD.alpha, :107-142): df.df, max|df|, df.df_last, df_last.df_last, s.y, s.s,
//             y.y and max|y| with s = x_last - x, y = df_last - df;
//   step      d = -df + beta d_last (or -df), x_new = x + alpha d (PGD.iter, :226-236);
//   project   the reference's bisection for the shift l of the projection
//             clip(xs + l dg, lo, hi) onto dg.x - vf <= 0 (project_to_feasible, :144-170),
//             for one constraint or for one constraint per block of the design (the
//             multi-material volume constraints, bisected in lockstep):
//             l1 = 0, l2 = -1e12, midpoint (l1 + l2) / 2, l2 = mid when the constraint holds
//             else l1 = mid, until (l2 - l1) / (l2 + l1) <= tol; the result is the design at
//             the last midpoint evaluated, or clip(xs) when that already satisfies it.
//             Like the OC update, a pass evaluates the constraint at the 31 midpoints of the
//             next five bisection levels and a one-block kernel replays the decisions.
// Every sum is a fixed-order two-stage reduction (run-to-run reproducible).
#include <cmath>

#include "common.cuh"

namespace pf {

constexpr int kPT = 256;
constexpr int kPgdTree = 31;
constexpr int kStats = 8;

static unsigned pgd_blocks(long long n) {
    long long nb = (n + kPT - 1) / kPT;
    if (nb > 2LL * kNumSM) nb = 2LL * kNumSM;
    return (unsigned)(nb < 1 ? 1 : nb);
}

__device__ __forceinline__ double block_max(double v, double* smem) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) smem[w] = v;
    __syncthreads();
    double m = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kPT / 32; i++) m = fmax(m, smem[i]);
    __syncthreads();
    return m;
}

// partials[b * kStats + q]: sums (q = 0, 2..6) and maxima (q = 1, 7) of block b
__global__ void __launch_bounds__(kPT) k_pgd_stats(long long n, const double* __restrict__ x, const double* __restrict__ df,
                                                   const double* __restrict__ xl, const double* __restrict__ dfl,
                                                   double* __restrict__ partials) {
    __shared__ double s_red[kPT / 32];
    double v[kStats] = {0, 0, 0, 0, 0, 0, 0, 0};
    const bool hist = xl != nullptr && dfl != nullptr;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double g = df[i];
        v[0] += g * g;
        v[1] = fmax(v[1], fabs(g));
        if (hist) {
            const double gl = dfl[i], s = xl[i] - x[i], y = gl - g;
            v[2] += g * gl;
            v[3] += gl * gl;
            v[4] += s * y;
            v[5] += s * s;
            v[6] += y * y;
            v[7] = fmax(v[7], fabs(y));
        }
    }
#pragma unroll
    for (int q = 0; q < kStats; q++) {
        const double r = (q == 1 || q == 7) ? block_max(v[q], s_red) : block_sum<kPT>(v[q], s_red);
        if (threadIdx.x == 0) partials[(long long)blockIdx.x * kStats + q] = r;
    }
}

__global__ void k_pgd_stats_final(const double* __restrict__ partials, int np, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= kStats) return;
    double r = 0.0;
    for (int b = 0; b < np; b++) {
        const double p = partials[(long long)b * kStats + q];
        r = (q == 1 || q == 7) ? fmax(r, p) : r + p;
    }
    out[q] = r;
}

__global__ void k_pgd_step(long long n, const double* __restrict__ x, const double* __restrict__ df,
                           const double* __restrict__ dl, double beta, double alpha, double* __restrict__ d,
                           double* __restrict__ xn) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double di = dl ? -df[i] + beta * dl[i] : -df[i];
        d[i] = di;
        xn[i] = x[i] + alpha * di;
    }
}

// ---- projection ---------------------------------------------------------------------------
// m volume constraints, one per block of the design (xs and dg hold m blocks of ne; dg's
// block c is row c of the constraint gradient restricted to block c, the only part of the
// row that is nonzero for MinimumCompliance).  The m bisections run in lockstep: a sweep
// moves every shift to its midpoint, and sweeps continue while ANY block's
// (l2 - l1) / (l2 + l1) exceeds tol (PGD.py:156-163).  A block whose clip(xs) is already
// feasible keeps l1 = 0 and its ratio at 1 until l2 underflows to zero (NaN ends it), so
// with m > 1 a run can take about 1100 sweeps.
constexpr int kPgdMaxBlocks = 8;
constexpr int kPgdChunk = 24;         // passes (5 sweeps each) between host checks
constexpr int kPgdMaxPasses = 240;    // 1200 sweeps: past the underflow of -1e12 / 2^k

struct PgdComp {
    double l1, l2, lmid, g0, g[kPgdTree], lam[kPgdTree];
};
struct PgdState {
    double tol;
    int done, steps, feasible0, nm;
    PgdComp c[kPgdMaxBlocks];
};
struct PgdVf {
    double v[kPgdMaxBlocks];
};

__device__ void pgd_tree(PgdComp* S) {
    // node t covers (a_t, b_t) = (l1, l2); left child (a_t, m_t) follows g(m_t) <= 0 (l2 = m_t)
    double a[kPgdTree], b[kPgdTree];
    a[0] = S->l1;
    b[0] = S->l2;
    for (int t = 0; t < kPgdTree; t++) {
        const double m = (a[t] + b[t]) / 2.0;
        S->lam[t] = m;
        if (2 * t + 2 < kPgdTree) {
            a[2 * t + 1] = a[t];
            b[2 * t + 1] = m;
            a[2 * t + 2] = m;
            b[2 * t + 2] = b[t];
        }
    }
}

__device__ __forceinline__ double pgd_x(double xs, double l, double d, double lo, double hi) {
    return fmin(fmax(xs + l * d, lo), hi);
}

__device__ __forceinline__ bool pgd_open(const PgdComp& c, double tol) { return (c.l2 - c.l1) / (c.l2 + c.l1) > tol; }

// g at l = 0, block c = blockIdx.y (partials[c * gridDim.x + b])
__global__ void __launch_bounds__(kPT) k_pgd_g0(long long ne, const double* __restrict__ xs, const double* __restrict__ dg,
                                                double lo, double hi, double* partials) {
    __shared__ double s_red[kPT / 32];
    const long long off = (long long)blockIdx.y * ne;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (long long)gridDim.x * blockDim.x)
        s += dg[off + i] * pgd_x(xs[off + i], 0.0, dg[off + i], lo, hi);
    s = block_sum<kPT>(s, s_red);
    if (threadIdx.x == 0) partials[(long long)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

__global__ void __launch_bounds__(kPT) k_pgd_init(const double* partials, int np, int nm, PgdVf vf, double tol,
                                                  PgdState* S) {
    __shared__ double s_red[kPT / 32];
    bool feasible = true;
    for (int c = 0; c < nm; c++) {
        double s = 0.0;
        for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[c * np + i];
        s = block_sum<kPT>(s, s_red);
        if (threadIdx.x == 0) {
            PgdComp& C = S->c[c];
            C.g0 = s - vf.v[c];
            C.l1 = 0.0;
            C.l2 = -1e12;
            C.lmid = 0.0;
            feasible = feasible && C.g0 <= 0.0;
            pgd_tree(&C);
        }
    }
    if (threadIdx.x == 0) {
        S->tol = tol;
        S->nm = nm;
        S->steps = 0;
        S->feasible0 = feasible;
        S->done = feasible;
    }
}

// the constraint at the 31 midpoints of the next five sweeps, block c = blockIdx.y
// (partials[(c * gridDim.x + b) * 31 + t])
__global__ void __launch_bounds__(kPT) k_pgd_eval(long long ne, const double* __restrict__ xs, const double* __restrict__ dg,
                                                  double lo, double hi, const PgdState* S, double* partials) {
    __shared__ double s_lam[kPgdTree];
    __shared__ double s_part[kPT / 32][kPgdTree];
    if (S->done) return;
    if (threadIdx.x < kPgdTree) s_lam[threadIdx.x] = S->c[blockIdx.y].lam[threadIdx.x];
    __syncthreads();
    const long long off = (long long)blockIdx.y * ne;
    double acc[kPgdTree];
#pragma unroll
    for (int t = 0; t < kPgdTree; t++) acc[t] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (long long)gridDim.x * blockDim.x) {
        const double x = xs[off + i], d = dg[off + i];
#pragma unroll
        for (int t = 0; t < kPgdTree; t++) acc[t] += d * pgd_x(x, s_lam[t], d, lo, hi);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < kPgdTree; t++) {
        const double v = warp_sum(acc[t]);
        if (l == 0) s_part[w][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < kPgdTree) {
        double s = 0.0;
        for (int k = 0; k < kPT / 32; k++) s += s_part[k][threadIdx.x];
        partials[((long long)blockIdx.y * gridDim.x + blockIdx.x) * kPgdTree + threadIdx.x] = s;
    }
}

// replays up to five lockstep sweeps from the evaluated midpoints
__global__ void __launch_bounds__(32) k_pgd_decide(const double* partials, int np, PgdVf vf, PgdState* S) {
    if (S->done) return;
    const int t = threadIdx.x, nm = S->nm;
    if (t < kPgdTree)
        for (int c = 0; c < nm; c++) {
            double s = 0.0;
            const double* pc = partials + (size_t)c * np * kPgdTree;
            for (int b = 0; b < np; b++) s += pc[(long long)b * kPgdTree + t];
            S->c[c].g[t] = s - vf.v[c];
        }
    __syncwarp();
    if (t == 0) {
        const double tol = S->tol;
        int node[kPgdMaxBlocks];
        for (int c = 0; c < nm; c++) node[c] = 0;
        bool done = false;
        for (int d = 0; d < 5; d++) {
            bool any = false;
            for (int c = 0; c < nm; c++) any |= pgd_open(S->c[c], tol);
            if (!any) {
                done = true;
                break;
            }
            S->steps += 1;
            for (int c = 0; c < nm; c++) {
                PgdComp& C = S->c[c];
                const double lmid = C.lam[node[c]];
                C.lmid = lmid;
                if (C.g[node[c]] <= 0.0) {
                    C.l2 = lmid;
                    node[c] = 2 * node[c] + 1;
                } else {
                    C.l1 = lmid;
                    node[c] = 2 * node[c] + 2;
                }
            }
        }
        if (!done) {
            bool any = false;
            for (int c = 0; c < nm; c++) any |= pgd_open(S->c[c], tol);
            done = !any;
        }
        S->done = done;
        if (!done)
            for (int c = 0; c < nm; c++) pgd_tree(&S->c[c]);
    }
}

__global__ void k_pgd_write(long long ne, const double* __restrict__ xs, const double* __restrict__ dg, double lo,
                            double hi, const PgdState* S, double* __restrict__ xn) {
    const double l = S->feasible0 ? 0.0 : S->c[blockIdx.y].lmid;
    const long long off = (long long)blockIdx.y * ne;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += (long long)gridDim.x * blockDim.x)
        xn[off + i] = pgd_x(xs[off + i], l, dg[off + i], lo, hi);
}

// blocks per design block: the grid over all m blocks stays within two waves
static unsigned pgd_blocks_per(long long ne, int nm) {
    long long nb = (ne + kPT - 1) / kPT;
    const long long cap = (2LL * kNumSM + nm - 1) / nm;
    if (nb > cap) nb = cap;
    return (unsigned)(nb < 1 ? 1 : nb);
}

static size_t pgd_project_workspace(long long ne, int nm) {
    return (size_t)pgd_blocks_per(ne, nm) * nm * kPgdTree + (sizeof(PgdState) + 7) / 8 + 8;
}

// h_out (host, may be NULL) = {steps, feasible at l = 0, l of block 0 .. l of block m-1}
static int pgd_project(long long ne, int nm, const double* xs, const double* dg, const PgdVf& vf, double lo, double hi,
                       double tol, double* x_new, double* work, double* h_out, cudaStream_t st) {
    const unsigned nb = pgd_blocks_per(ne, nm);
    double* partials = work;
    PgdState* S = reinterpret_cast<PgdState*>(work + (size_t)nb * nm * kPgdTree);
    const dim3 grid(nb, (unsigned)nm);
    count_launch(2);
    k_pgd_g0<<<grid, kPT, 0, st>>>(ne, xs, dg, lo, hi, partials);
    k_pgd_init<<<1, kPT, 0, st>>>(partials, (int)nb, nm, vf, tol, S);
    PgdState h;
    h.done = 0;
    for (int pass = 0; pass < kPgdMaxPasses && !h.done;) {
        for (int p = 0; p < kPgdChunk; p++, pass++) {
            count_launch(2);
            k_pgd_eval<<<grid, kPT, 0, st>>>(ne, xs, dg, lo, hi, S, partials);
            k_pgd_decide<<<1, 32, 0, st>>>(partials, (int)nb, vf, S);
        }
        PF_LAUNCH_CHECK("pgd project launch");
        if (!h_out) break;  // no host synchronisation: one chunk (120 sweeps)
        PF_CUDA(cudaMemcpyAsync(&h, S, sizeof(PgdState), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaStreamSynchronize(st));
    }
    count_launch();
    k_pgd_write<<<dim3(nb * 4, (unsigned)nm), kPT, 0, st>>>(ne, xs, dg, lo, hi, S, x_new);
    PF_LAUNCH_CHECK("pgd write launch");
    if (h_out) {
        h_out[0] = (double)h.steps;
        h_out[1] = (double)h.feasible0;
        for (int c = 0; c < nm; c++) h_out[2 + c] = h.feasible0 ? 0.0 : h.c[c].lmid;
        if (!h.done) return fail(PF_NOT_CONVERGED, "PGD projection bisection did not terminate in %d sweeps", h.steps);
    }
    return PF_OK;
}

}  // namespace pf

using namespace pf;

extern "C" size_t pf_pgd_workspace_size(long long n) {
    const long long nb = pgd_blocks(n < 1 ? 1 : n);
    return (size_t)(nb * kStats + kStats) + pgd_project_workspace(n < 1 ? 1 : n, 1);
}

extern "C" size_t pf_pgd_multi_workspace_size(long long ne, int nm) {
    if (nm < 1 || nm > kPgdMaxBlocks) return 0;
    return pgd_project_workspace(ne < 1 ? 1 : ne, nm);
}

extern "C" int pf_pgd_stats_f64(long long n, const double* x, const double* df, const double* x_last,
                                const double* df_last, double* work, double* h_out, void* stream) {
    if (n < 1 || !x || !df || !work || !h_out) return fail(PF_BAD_ARG, "pf_pgd_stats_f64: bad argument");
    if ((x_last == nullptr) != (df_last == nullptr))
        return fail(PF_BAD_ARG, "pf_pgd_stats_f64: x_last and df_last are both given or both NULL");
    cudaStream_t st = as_stream(stream);
    const unsigned nb = pgd_blocks(n);
    double* partials = work;
    double* out = work + (size_t)nb * kStats;
    count_launch(2);
    k_pgd_stats<<<nb, kPT, 0, st>>>(n, x, df, x_last, df_last, partials);
    k_pgd_stats_final<<<1, 32, 0, st>>>(partials, (int)nb, out);
    PF_LAUNCH_CHECK("pgd stats launch");
    PF_CUDA(cudaMemcpyAsync(h_out, out, kStats * sizeof(double), cudaMemcpyDeviceToHost, st));
    PF_CUDA(cudaStreamSynchronize(st));
    return PF_OK;
}

extern "C" int pf_pgd_step_f64(long long n, const double* x, const double* df, const double* d_last, double beta,
                               double alpha, double* d, double* x_new, void* stream) {
    if (n < 1 || !x || !df || !d || !x_new) return fail(PF_BAD_ARG, "pf_pgd_step_f64: bad argument");
    count_launch();
    k_pgd_step<<<pgd_blocks(n) * 4, kPT, 0, as_stream(stream)>>>(n, x, df, d_last, beta, alpha, d, x_new);
    PF_LAUNCH_CHECK("pgd step launch");
    return PF_OK;
}

extern "C" int pf_pgd_project_f64(long long n, const double* xs, const double* dg, double vf, double lo, double hi,
                                  double tol, double* x_new, double* work, double* h_out, void* stream) {
    if (n < 1 || !xs || !dg || !x_new || !work || !(tol > 0.0) || !(lo <= hi))
        return fail(PF_BAD_ARG, "pf_pgd_project_f64: bad argument");
    PgdVf v;
    v.v[0] = vf;
    double h[3];
    const int rc = pgd_project(n, 1, xs, dg, v, lo, hi, tol, x_new, work, h_out ? h : nullptr, as_stream(stream));
    if (h_out) {
        h_out[0] = h[2];
        h_out[1] = h[0];
        h_out[2] = h[1];
    }
    return rc;
}

extern "C" int pf_pgd_project_multi_f64(long long ne, int nm, const double* xs, const double* dg, const double* h_vf,
                                        double lo, double hi, double tol, double* x_new, double* work, double* h_out,
                                        void* stream) {
    if (ne < 1 || nm < 1 || nm > kPgdMaxBlocks || !xs || !dg || !h_vf || !x_new || !work || !h_out || !(tol > 0.0) ||
        !(lo <= hi))
        return fail(PF_BAD_ARG, "pf_pgd_project_multi_f64: bad argument (1..%d blocks, h_out required)",
                    kPgdMaxBlocks);
    PgdVf v;
    for (int c = 0; c < nm; c++) v.v[c] = h_vf[c];
    return pgd_project(ne, nm, xs, dg, v, lo, hi, tol, x_new, work, h_out, as_stream(stream));
}
