// SIMP element-wise steps, deterministic reductions and the OC update.
//
// penalize / penalize_grad follow pyFANTOM/Problem/CUDA/MinimumCompliance.py:305-324 and
// :351-367 (single material): optional Heaviside projection
//   H(r) = (tanh(b eta) + tanh(b (r - eta))) / (tanh(b eta) + tanh(b (1 - eta))),
//   E = clip(clip(H^p, void, 1) * E_mul, void, inf),   dE = p H^(p-1) H'(r) E_mul.
//
// OC (pyFANTOM/Optimizers/CUDA/OC.py:67-129) bisects the Lagrange multiplier with the host
// testing g(x_new) after every step.  Here a pass evaluates the constraint at all 31
// midpoints of the next five levels of the bisection tree in one sweep over the elements
// (one partial sum per midpoint and block), and a one-block kernel replays the five
// sequential decisions with the reference's stopping rule; the midpoints are formed
// exactly as the sequential loop forms them, so the sequence of (l1, l2) is the same.
#include <cmath>

#include <vector>

#include "common.cuh"

namespace pf {

constexpr int kRT = 256;

__device__ __forceinline__ void heavy(double r, double beta, double eta, double* h, double* dh) {
    const double den = tanh(beta * eta) + tanh(beta * (1.0 - eta));
    const double t = tanh(beta * (r - eta));
    *h = (tanh(beta * eta) + t) / den;
    *dh = beta * (1.0 - t * t) / den;
}

__global__ void k_penalize(long long n, const double* __restrict__ rho, pf_simp_params P, double* __restrict__ E,
                           double* __restrict__ dE) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double r = rho[i], dh = 1.0;
        if (P.heavyside) heavy(rho[i], P.beta, P.eta, &r, &dh);
        if (E) {
            double e = pow(r, P.penalty);
            e = fmin(fmax(e, P.void_value), 1.0) * P.E_mul;
            E[i] = fmax(e, P.void_value);
        }
        if (dE) dE[i] = P.penalty * pow(r, P.penalty - 1.0) * dh * P.E_mul;
    }
}

// Multi-material SIMP (pyFANTOM/Problem/CUDA/MinimumCompliance.py:326-349, 369-411): with
// a_i = H(rho_i)^p and b_i = 1 - a_i,
//   E = max(sum_i E_mul_i a_i prod_{j != i} b_j, void)
//   dE/drho_k = H'(rho_k) sum_i E_mul_i { p H^(p-1)(rho_k) prod_{j != k} b_j            (i = k)
//                                         -p H^(p-1)(rho_k) a_i prod_{j != i, k} b_j     (i != k) }
// rho and dE are material-major [n_material][n_elements] (the design-variable order).
constexpr int kMaxMaterials = 8;
struct MultiEmul {
    double v[kMaxMaterials];
};
__global__ void k_penalize_multi(long long ne, int nm, const double* __restrict__ rho, pf_simp_params P, MultiEmul em,
                                 double* __restrict__ E, double* __restrict__ dE) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
        double a[kMaxMaterials], b[kMaxMaterials], da[kMaxMaterials];
        for (int k = 0; k < nm; k++) {
            double r = rho[k * ne + e], dh = 1.0;
            if (P.heavyside) heavy(rho[k * ne + e], P.beta, P.eta, &r, &dh);
            a[k] = pow(r, P.penalty);
            b[k] = 1.0 - a[k];
            da[k] = P.penalty * pow(r, P.penalty - 1.0) * dh;
        }
        if (E) {
            double s = 0.0;
            for (int i = 0; i < nm; i++) {
                double t = a[i];
                for (int j = 0; j < nm; j++)
                    if (j != i) t *= b[j];
                s += em.v[i] * t;
            }
            E[e] = fmax(s, P.void_value);
        }
        if (dE) {
            for (int k = 0; k < nm; k++) {
                double s = 0.0;
                for (int i = 0; i < nm; i++) {
                    double t = i == k ? da[k] : -da[k] * a[i];
                    for (int j = 0; j < nm; j++)
                        if (j != i && j != k) t *= b[j];
                    s += em.v[i] * t;
                }
                dE[k * ne + e] = s;
            }
        }
    }
}

__global__ void k_mul(long long n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = a[i] * b[i];
}

static unsigned grid_for(long long n) {
    long long nb = (n + kRT - 1) / kRT;
    if (nb > 8LL * kNumSM) nb = 8LL * kNumSM;
    return (unsigned)(nb < 1 ? 1 : nb);
}

__global__ void __launch_bounds__(kRT) k_dot_part(long long n, const double* __restrict__ a, const double* __restrict__ b,
                                                  double* partials) {
    __shared__ double s_red[kRT / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRT) k_sum_to(const double* partials, int np, double* out) {
    __shared__ double s_red[kRT / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------------------
// OC
// ---------------------------------------------------------------------------------------
constexpr int kOcTree = 31;  // midpoints of 5 bisection levels
constexpr int kOcPasses = 24;

struct OcState {
    double l1, l2, lmid, abs_sum, change2, g[kOcTree], lam[kOcTree];
    int done, steps, allzero, pad;
};

__global__ void __launch_bounds__(kRT) k_oc_prep(long long n, const double* __restrict__ x, const double* __restrict__ df,
                                                 const double* __restrict__ dg, double* __restrict__ ocp,
                                                 double* partials) {
    __shared__ double s_red[kRT / 32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double t = fmax(-df[i] / dg[i], 0.0);
        double q = sqrt(t);
        if (q != q) q = 0.0;
        const double v = x[i] * q;
        ocp[i] = v;
        s += fabs(v);
    }
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__device__ void oc_tree(OcState* S) {
    // heap layout: node t covers (a_t, b_t); its midpoint is (a_t + b_t) / 2; the left
    // child (a_t, m_t) follows g(m_t) <= 0 (l2 = m_t), the right child (m_t, b_t) otherwise
    double a[kOcTree], b[kOcTree];
    a[0] = S->l1;
    b[0] = S->l2;
    for (int t = 0; t < kOcTree; t++) {
        const double m = (a[t] + b[t]) / 2.0;
        S->lam[t] = m;
        if (2 * t + 2 < kOcTree) {
            a[2 * t + 1] = a[t];
            b[2 * t + 1] = m;
            a[2 * t + 2] = m;
            b[2 * t + 2] = b[t];
        }
    }
}

__global__ void __launch_bounds__(kRT) k_oc_init(const double* partials, int np, OcState* S) {
    __shared__ double s_red[kRT / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) {
        S->abs_sum = s;
        S->allzero = s == 0.0;
        S->l1 = 1e-9;
        S->l2 = 1e9;
        S->lmid = 0.0;
        S->done = 0;
        S->steps = 0;
        S->change2 = 0.0;
        oc_tree(S);
    }
}

__device__ __forceinline__ double oc_xnew(double xi, double oc, double lam, double move) {
    const double xu = fmin(fmax(xi + move, 0.0), 1.0), xl = fmin(fmax(xi - move, 0.0), 1.0);
    return fmax(0.0, fmax(xl, fmin(1.0, fmin(xu, oc / lam))));
}

__global__ void __launch_bounds__(kRT) k_oc_eval(long long n, const double* __restrict__ x, const double* __restrict__ ocp,
                                                 const double* __restrict__ dg, double move, const OcState* S,
                                                 double* partials) {
    __shared__ double s_lam[kOcTree];
    __shared__ double s_part[kRT / 32][kOcTree];
    if (S->done) return;
    if (threadIdx.x < kOcTree) s_lam[threadIdx.x] = S->lam[threadIdx.x];
    __syncthreads();
    const bool allzero = S->allzero;
    double acc[kOcTree];
#pragma unroll
    for (int t = 0; t < kOcTree; t++) acc[t] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double xi = x[i], oc = allzero ? 1e-3 : ocp[i], d = dg[i];
#pragma unroll
        for (int t = 0; t < kOcTree; t++) acc[t] += d * oc_xnew(xi, oc, s_lam[t], move);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < kOcTree; t++) {
        const double v = warp_sum(acc[t]);
        if (l == 0) s_part[w][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < kOcTree) {
        double s = 0.0;
        for (int k = 0; k < kRT / 32; k++) s += s_part[k][threadIdx.x];
        partials[(long long)blockIdx.x * kOcTree + threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(32) k_oc_step(const double* partials, int np, double vf, OcState* S) {
    if (S->done) return;
    const int t = threadIdx.x;
    if (t < kOcTree) {
        double s = 0.0;
        for (int b = 0; b < np; b++) s += partials[(long long)b * kOcTree + t];
        S->g[t] = s - vf;
    }
    __syncwarp();
    if (t == 0) {
        int node = 0;
        for (int d = 0; d < 5; d++) {
            const double l1 = S->l1, l2 = S->l2;
            if (!((l2 - l1) / (l2 + l1) > 1e-8)) {
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
            if (!((l2 - l1) / (l2 + l1) > 1e-8))
                S->done = 1;
            else
                oc_tree(S);
        }
    }
}

__global__ void __launch_bounds__(kRT) k_oc_write(long long n, const double* __restrict__ x, const double* __restrict__ ocp,
                                                  double move, const OcState* S, double* __restrict__ xnew,
                                                  double* partials) {
    __shared__ double s_red[kRT / 32];
    const double lam = S->lmid;
    const bool allzero = S->allzero;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = oc_xnew(x[i], allzero ? 1e-3 : ocp[i], lam, move);
        xnew[i] = v;
        const double d = x[i] - v;
        s += d * d;
    }
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRT) k_oc_change(const double* partials, int np, OcState* S) {
    __shared__ double s_red[kRT / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) S->change2 = s;
}

// Several volume constraints (one per material, variables material-major): the reference
// bisects all multipliers in lockstep while any of them is unconverged (OC.py:111-127),
// so every multiplier takes the same number of steps.  One OcState per material; the
// evaluation pass runs per material segment, this kernel replays the lockstep decisions.
struct MultiVf {
    double v[kMaxMaterials];
};
__global__ void __launch_bounds__(32) k_oc_step_multi(const double* partials, int np, int nm, MultiVf vf, OcState* S) {
    if (S[0].done) return;
    const int t = threadIdx.x;
    for (int k = 0; k < nm; k++) {
        if (t < kOcTree) {
            double s = 0.0;
            const double* pk = partials + (size_t)k * np * kOcTree;
            for (int b = 0; b < np; b++) s += pk[(long long)b * kOcTree + t];
            S[k].g[t] = s - vf.v[k];
        }
    }
    __syncwarp();
    if (t == 0) {
        int node[kMaxMaterials];
        for (int k = 0; k < nm; k++) node[k] = 0;
        bool done = false;
        for (int d = 0; d < 5 && !done; d++) {
            bool any = false;
            for (int k = 0; k < nm; k++) any |= (S[k].l2 - S[k].l1) / (S[k].l2 + S[k].l1) > 1e-8;
            if (!any) {
                done = true;
                break;
            }
            for (int k = 0; k < nm; k++) {
                const double lmid = S[k].lam[node[k]];
                S[k].lmid = lmid;
                S[k].steps += 1;
                if (S[k].g[node[k]] <= 0.0) {
                    S[k].l2 = lmid;
                    node[k] = 2 * node[k] + 1;
                } else {
                    S[k].l1 = lmid;
                    node[k] = 2 * node[k] + 2;
                }
            }
        }
        if (!done) {
            bool any = false;
            for (int k = 0; k < nm; k++) any |= (S[k].l2 - S[k].l1) / (S[k].l2 + S[k].l1) > 1e-8;
            done = !any;
        }
        for (int k = 0; k < nm; k++) {
            S[k].done = done;
            if (!done) oc_tree(&S[k]);
        }
    }
}

__global__ void __launch_bounds__(kRT) k_oc_init_multi(const double* partials, int np, int nm, OcState* S) {
    __shared__ double s_red[kRT / 32];
    double s = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
    s = block_sum<kRT>(s, s_red);
    if (threadIdx.x == 0) {
        for (int k = 0; k < nm; k++) {
            S[k].abs_sum = s;
            S[k].allzero = s == 0.0;
            S[k].l1 = 1e-9;
            S[k].l2 = 1e9;
            S[k].lmid = 0.0;
            S[k].done = 0;
            S[k].steps = 0;
            S[k].change2 = 0.0;
            oc_tree(&S[k]);
        }
    }
}

static unsigned oc_blocks(long long n) {
    long long nb = (n + kRT - 1) / kRT;
    if (nb > 2LL * kNumSM) nb = 2LL * kNumSM;
    return (unsigned)(nb < 1 ? 1 : nb);
}

size_t oc_workspace(long long n) {
    return (size_t)n + (size_t)oc_blocks(n) * kOcTree + (sizeof(OcState) + 7) / 8 + 8;
}

int oc_update(long long n, const double* x, const double* df, const double* dg, double vf, double move,
              double* x_new, double* work, double* h_out, cudaStream_t st) {
    const unsigned nb = oc_blocks(n);
    double* ocp = work;
    double* partials = work + n;
    OcState* S = reinterpret_cast<OcState*>(partials + (size_t)nb * kOcTree);
    pf::count_launch();
    k_oc_prep<<<nb, kRT, 0, st>>>(n, x, df, dg, ocp, partials);
    pf::count_launch();
    k_oc_init<<<1, kRT, 0, st>>>(partials, nb, S);
    for (int p = 0; p < kOcPasses; p++) {
        pf::count_launch();
        k_oc_eval<<<nb, kRT, 0, st>>>(n, x, ocp, dg, move, S, partials);
        pf::count_launch();
        k_oc_step<<<1, 32, 0, st>>>(partials, nb, vf, S);
    }
    pf::count_launch();
    k_oc_write<<<nb, kRT, 0, st>>>(n, x, ocp, move, S, x_new, partials);
    pf::count_launch();
    k_oc_change<<<1, kRT, 0, st>>>(partials, nb, S);
    PF_LAUNCH_CHECK("oc launch");
    if (h_out) {
        OcState h;
        PF_CUDA(cudaMemcpyAsync(&h, S, sizeof(OcState), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaStreamSynchronize(st));
        h_out[0] = sqrt(h.change2);
        h_out[1] = h.lmid;
        h_out[2] = (double)h.steps;
        if (!h.done) return fail(PF_NOT_CONVERGED, "OC bisection did not terminate in %d steps", h.steps);
    }
    return PF_OK;
}

size_t oc_multi_workspace(long long ne, int nm) {
    const long long n = ne * nm;
    return (size_t)n + (size_t)oc_blocks(ne) * kOcTree * nm + (size_t)oc_blocks(n) +
           (sizeof(OcState) * nm + 7) / 8 + 8;
}

int oc_update_multi(long long ne, int nm, const double* x, const double* df, const double* dg, const double* vf,
                    double move, double* x_new, double* work, double* h_out, cudaStream_t st) {
    const long long n = ne * nm;
    const unsigned nb = oc_blocks(ne), nbn = oc_blocks(n);
    double* ocp = work;
    double* partials = work + n;                               // nm segments of nb * kOcTree
    double* sums = partials + (size_t)nb * kOcTree * nm;        // nbn
    OcState* S = reinterpret_cast<OcState*>(sums + nbn);
    MultiVf mv;
    for (int k = 0; k < nm; k++) mv.v[k] = vf[k];
    pf::count_launch(2);
    k_oc_prep<<<nbn, kRT, 0, st>>>(n, x, df, dg, ocp, sums);
    k_oc_init_multi<<<1, kRT, 0, st>>>(sums, nbn, nm, S);
    for (int p = 0; p < kOcPasses; p++) {
        for (int k = 0; k < nm; k++) {
            pf::count_launch();
            k_oc_eval<<<nb, kRT, 0, st>>>(ne, x + k * ne, ocp + k * ne, dg + k * ne, move, &S[k],
                                          partials + (size_t)k * nb * kOcTree);
        }
        pf::count_launch();
        k_oc_step_multi<<<1, 32, 0, st>>>(partials, nb, nm, mv, S);
    }
    for (int k = 0; k < nm; k++) {
        pf::count_launch();
        k_oc_write<<<nb, kRT, 0, st>>>(ne, x + k * ne, ocp + k * ne, move, &S[k], x_new + k * ne,
                                       partials + (size_t)k * nb * kOcTree);
    }
    PF_LAUNCH_CHECK("oc multi launch");
    if (h_out) {  // change^2: the per-block sums k_oc_write left in each material's segment
        std::vector<OcState> h(nm);
        std::vector<double> part((size_t)nb * kOcTree * nm);
        PF_CUDA(cudaMemcpyAsync(h.data(), S, sizeof(OcState) * nm, cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaMemcpyAsync(part.data(), partials, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st));
        PF_CUDA(cudaStreamSynchronize(st));
        double c2 = 0.0;
        for (int k = 0; k < nm; k++)
            for (unsigned b = 0; b < nb; b++) c2 += part[(size_t)k * nb * kOcTree + b];
        h_out[0] = sqrt(c2);
        h_out[1] = h[0].lmid;
        h_out[2] = (double)h[0].steps;
        if (!h[0].done) return fail(PF_NOT_CONVERGED, "OC bisection did not terminate in %d steps", h[0].steps);
    }
    return PF_OK;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_penalize_multi_f64(long long ne, int nm, const double* rho, const pf_simp_params* p,
                                     const double* h_E_mul, double* E, double* dE, void* stream) {
    if (ne < 0 || nm < 2 || nm > kMaxMaterials || !rho || !p || !h_E_mul || (!E && !dE))
        return fail(PF_BAD_ARG, "pf_penalize_multi_f64: bad argument (2..%d materials)", kMaxMaterials);
    MultiEmul em;
    for (int k = 0; k < nm; k++) em.v[k] = h_E_mul[k];
    count_launch();
    k_penalize_multi<<<grid_for(ne < 1 ? 1 : ne), kRT, 0, as_stream(stream)>>>(ne, nm, rho, *p, em, E, dE);
    PF_LAUNCH_CHECK("penalize multi launch");
    return PF_OK;
}

extern "C" size_t pf_oc_multi_workspace_size(long long ne, int nm) { return oc_multi_workspace(ne < 1 ? 1 : ne, nm); }

extern "C" int pf_oc_update_multi_f64(long long ne, int nm, const double* x, const double* df, const double* dg,
                                      const double* h_vf, double move, double* x_new, double* work, double* h_out,
                                      void* stream) {
    if (ne < 1 || nm < 1 || nm > kMaxMaterials || !x || !df || !dg || !h_vf || !x_new || !work)
        return fail(PF_BAD_ARG, "pf_oc_update_multi_f64: bad argument (1..%d materials)", kMaxMaterials);
    return oc_update_multi(ne, nm, x, df, dg, h_vf, move, x_new, work, h_out, as_stream(stream));
}

extern "C" int pf_penalize_f64(long long n, const double* rho, const pf_simp_params* p, double* E, double* dE,
                               void* stream) {
    if (n < 0 || !rho || !p || (!E && !dE)) return fail(PF_BAD_ARG, "pf_penalize_f64: bad argument");
    if (n == 0) return PF_OK;
    pf::count_launch();
    k_penalize<<<grid_for(n), kRT, 0, as_stream(stream)>>>(n, rho, *p, E, dE);
    PF_LAUNCH_CHECK("penalize launch");
    return PF_OK;
}

extern "C" int pf_mul_f64(long long n, const double* a, const double* b, double* out, void* stream) {
    if (n < 0 || !a || !b || !out) return fail(PF_BAD_ARG, "pf_mul_f64: bad argument");
    if (n == 0) return PF_OK;
    pf::count_launch();
    k_mul<<<grid_for(n), kRT, 0, as_stream(stream)>>>(n, a, b, out);
    PF_LAUNCH_CHECK("mul launch");
    return PF_OK;
}

extern "C" size_t pf_dot_workspace_size(long long n) { return (size_t)grid_for(n < 1 ? 1 : n) + 1; }

extern "C" int pf_dot_f64(long long n, const double* a, const double* b, double* result, double* work, void* stream) {
    if (n < 0 || !a || !b || !result || !work) return fail(PF_BAD_ARG, "pf_dot_f64: bad argument");
    cudaStream_t st = as_stream(stream);
    const unsigned nb = grid_for(n < 1 ? 1 : n);
    pf::count_launch();
    k_dot_part<<<nb, kRT, 0, st>>>(n, a, b, work);
    pf::count_launch();
    k_sum_to<<<1, kRT, 0, st>>>(work, (int)nb, result);
    PF_LAUNCH_CHECK("dot launch");
    return PF_OK;
}

extern "C" size_t pf_oc_workspace_size(long long n) { return oc_workspace(n < 1 ? 1 : n); }

extern "C" int pf_oc_update_f64(long long n, const double* x, const double* df, const double* dg, double vf, double move,
                                double* x_new, double* work, double* h_out, void* stream) {
    if (n < 1 || !x || !df || !dg || !x_new || !work) return fail(PF_BAD_ARG, "pf_oc_update_f64: bad argument");
    if (!(move >= 0.0)) return fail(PF_BAD_ARG, "move must be >= 0");
    return oc_update(n, x, df, dg, vf, move, x_new, work, h_out, as_stream(stream));
}
