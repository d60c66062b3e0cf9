// Projected gradient descent (pyFANTOM/Optimizers/CUDA/PGD.py:6-372), single volume
// constraint: the vector work of one iteration.
//
//   stats     one pass over (x, df, x_last, df_last) for the scalars of the step-size rule
//             (PGD.alpha, :107-142): df.df, max|df|, df.df_last, df_last.df_last, s.y, s.s,
//             y.y and max|y| with s = x_last - x, y = df_last - df;
//   step      d = -df + beta d_last (or -df), x_new = x + alpha d (PGD.iter, :226-236);
//   project   the reference's bisection for the shift l of the projection
//             clip(xs + l dg, lo, hi) onto dg.x - vf <= 0 (project_to_feasible, :144-170):
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
constexpr int kPgdPasses = 24;
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
struct PgdState {
    double l1, l2, lmid, tol, g0, g[kPgdTree], lam[kPgdTree];
    int done, steps, feasible0, pad;
};

__device__ void pgd_tree(PgdState* S) {
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

// g at l = 0 (partials per block)
__global__ void __launch_bounds__(kPT) k_pgd_g0(long long n, const double* __restrict__ xs, const double* __restrict__ dg,
                                                double lo, double hi, double* partials) {
    __shared__ double s_red[kPT / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += dg[i] * pgd_x(xs[i], 0.0, dg[i], lo, hi);
    s = block_sum<kPT>(s, s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kPT) k_pgd_init(const double* partials, int np, double vf, double tol, PgdState* S) {
    __shared__ double s_red[kPT / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum<kPT>(s, s_red);
    if (threadIdx.x == 0) {
        S->g0 = s - vf;
        S->l1 = 0.0;
        S->l2 = -1e12;
        S->lmid = 0.0;
        S->tol = tol;
        S->steps = 0;
        S->feasible0 = S->g0 <= 0.0;
        S->done = S->feasible0;
        pgd_tree(S);
    }
}

__global__ void __launch_bounds__(kPT) k_pgd_eval(long long n, const double* __restrict__ xs, const double* __restrict__ dg,
                                                  double lo, double hi, const PgdState* S, double* partials) {
    __shared__ double s_lam[kPgdTree];
    __shared__ double s_part[kPT / 32][kPgdTree];
    if (S->done) return;
    if (threadIdx.x < kPgdTree) s_lam[threadIdx.x] = S->lam[threadIdx.x];
    __syncthreads();
    double acc[kPgdTree];
#pragma unroll
    for (int t = 0; t < kPgdTree; t++) acc[t] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double x = xs[i], d = dg[i];
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
        partials[(long long)blockIdx.x * kPgdTree + threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(32) k_pgd_decide(const double* partials, int np, double vf, PgdState* S) {
    if (S->done) return;
    const int t = threadIdx.x;
    if (t < kPgdTree) {
        double s = 0.0;
        for (int b = 0; b < np; b++) s += partials[(long long)b * kPgdTree + t];
        S->g[t] = s - vf;
    }
    __syncwarp();
    if (t == 0) {
        int node = 0;
        for (int d = 0; d < 5; d++) {
            const double l1 = S->l1, l2 = S->l2;
            if (!((l2 - l1) / (l2 + l1) > S->tol)) {
                S->done = 1;
                break;
            }
            const double lmid = S->lam[node];
            S->lmid = lmid;
            S->steps += 1;
            if (S->g[node] <= 0.0) {
                S->l2 = lmid;
                node = 2 * node + 1;
            } else {
                S->l1 = lmid;
                node = 2 * node + 2;
            }
        }
        if (!S->done) {
            const double l1 = S->l1, l2 = S->l2;
            if (!((l2 - l1) / (l2 + l1) > S->tol))
                S->done = 1;
            else
                pgd_tree(S);
        }
    }
}

__global__ void k_pgd_write(long long n, const double* __restrict__ xs, const double* __restrict__ dg, double lo,
                            double hi, const PgdState* S, double* __restrict__ xn) {
    const double l = S->feasible0 ? 0.0 : S->lmid;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        xn[i] = pgd_x(xs[i], l, dg[i], lo, hi);
}

}  // namespace pf

using namespace pf;

extern "C" size_t pf_pgd_workspace_size(long long n) {
    const long long nb = pgd_blocks(n < 1 ? 1 : n);
    return (size_t)(nb * kPgdTree + nb * kStats + kStats) + (sizeof(PgdState) + 7) / 8 + 8;
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
    cudaStream_t st = as_stream(stream);
    const unsigned nb = pgd_blocks(n);
    double* partials = work;
    PgdState* S = reinterpret_cast<PgdState*>(work + (size_t)nb * kPgdTree + (size_t)nb * kStats + kStats);
    count_launch(2);
    k_pgd_g0<<<nb, kPT, 0, st>>>(n, xs, dg, lo, hi, partials);
    k_pgd_init<<<1, kPT, 0, st>>>(partials, (int)nb, vf, tol, S);
    for (int p = 0; p < kPgdPasses; p++) {
        count_launch(2);
        k_pgd_eval<<<nb, kPT, 0, st>>>(n, xs, dg, lo, hi, S, partials);
        k_pgd_decide<<<1, 32, 0, st>>>(partials, (int)nb, vf, S);
    }
    count_launch();
    k_pgd_write<<<nb * 4, kPT, 0, st>>>(n, xs, dg, lo, hi, S, x_new);
    PF_LAUNCH_CHECK("pgd project launch");
    if (h_out) {
        PgdState h;
        PF_CUDA(cudaMemcpyAsync(&h, S, sizeof(PgdState), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaStreamSynchronize(st));
        h_out[0] = h.feasible0 ? 0.0 : h.lmid;
        h_out[1] = (double)h.steps;
        h_out[2] = (double)h.feasible0;
        if (!h.done) return fail(PF_NOT_CONVERGED, "PGD projection bisection did not terminate in %d steps", h.steps);
    }
    return PF_OK;
}
