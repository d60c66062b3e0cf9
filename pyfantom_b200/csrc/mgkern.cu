// Multigrid level kernels: grid transfers, Galerkin coarse operators, block-stencil
// matvec with the shared epilogues, stencil diagonal and dense export of the coarsest
// operator.  All kernels are generic over the dimension (DIM = 2 or 3, dof = DIM).
//
// Transfer operators follow the reference (pyFANTOM/core/CUDA/Kernels/mgm.cu:1-244):
// restriction R = diag(1/tw) Phat^T and prolongation P = Phat diag(1/tw) = R^T, where Phat
// is trilinear (bilinear) interpolation (weights 0.5^{|d|_1} on the 3^DIM fine nodes
// around an even fine node) and tw(c) = prod over axes of (1.5 on a boundary, else 2).
// Coarse grids floor nel / 2; along an axis with an odd element count the last fine node
// has one coarse parent, which the prolongation copies (there P differs from R^T, while
// the Galerkin product uses R^T throughout, as the reference).
// Coarse operators are Galerkin R A P with A_fine = Z K Z + I - Z on level 0
// (mgm.cu:247-447) and R A_l P on deeper levels (mgm.cu:449-590).
#include "common.cuh"
#include "elemop.cuh"
#include "mgkern.cuh"

namespace pf {

template <int DIM>
struct GridDev {
    int nel[3];
    int nn[3];
    long long n_nodes;
};

template <int DIM>
__host__ __device__ __forceinline__ long long nidx(const GridDev<DIM>& g, int i, int j, int k) {
    if (DIM == 3) return (long long)k + (long long)g.nn[2] * (i + (long long)g.nn[0] * j);
    return (long long)i + (long long)g.nn[0] * j;
}
// node index -> (i, j, k); 32-bit unsigned division (grids hold fewer than 2^31 DOFs,
// checked by validate_grid), far cheaper than the emulated 64-bit one
template <int DIM>
__device__ __forceinline__ void ndec(const GridDev<DIM>& g, long long n, int& i, int& j, int& k) {
    const unsigned un = (unsigned)n;
    if (DIM == 3) {
        const unsigned nz = (unsigned)g.nn[2], nx = (unsigned)g.nn[0];
        const unsigned t = un / nz;
        k = (int)(un - t * nz);
        j = (int)(t / nx);
        i = (int)(t - (unsigned)j * nx);
    } else {
        const unsigned nx = (unsigned)g.nn[0];
        j = (int)(un / nx);
        i = (int)(un - (unsigned)j * nx);
        k = 0;
    }
}
template <int DIM>
__device__ __forceinline__ bool nok(const GridDev<DIM>& g, int i, int j, int k) {
    if (i < 0 || j < 0 || i >= g.nn[0] || j >= g.nn[1]) return false;
    if (DIM == 3 && (k < 0 || k >= g.nn[2])) return false;
    return true;
}
template <int DIM>
__device__ __forceinline__ double total_weight(const GridDev<DIM>& gc, int i, int j, int k) {
    double t = ((i == 0 || i == gc.nn[0] - 1) ? 1.5 : 2.0) * ((j == 0 || j == gc.nn[1] - 1) ? 1.5 : 2.0);
    if (DIM == 3) t *= (k == 0 || k == gc.nn[2] - 1) ? 1.5 : 2.0;
    return t;
}
__device__ __forceinline__ double half_pow(int d) { return d == 0 ? 1.0 : d == 1 ? 0.5 : d == 2 ? 0.25 : 0.125; }

template <int DIM>
static GridDev<DIM> gdev(const Grid& g) {
    GridDev<DIM> d;
    for (int a = 0; a < 3; a++) {
        d.nel[a] = g.nel[a];
        d.nn[a] = g.nn[a];
    }
    d.n_nodes = g.n_nodes;
    return d;
}

// ---------------------------------------------------------------------------------------
// transfers
// ---------------------------------------------------------------------------------------
// One thread per (coarse node, component): the 3^DIM weighted fine values of that
// component, accumulated in the output precision.  Per axis the weights are 0.5 / 1 / 0.5
// and 1/tw factorises into 1/1.5 (boundary node) or 1/2.
template <int DIM, typename TI, typename TO>
__global__ void k_restrict(GridDev<DIM> gf, GridDev<DIM> gc, const TI* __restrict__ vf, TO* __restrict__ vc,
                           const int* skip, Jacobi0<TO> j0) {
    pdl_wait();
    pdl_trigger();
    using TA = TO;  // accumulation precision
    if (skip && *skip) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= gc.n_nodes * DIM) return;
    const long long c = (unsigned)t / DIM;
    const int d = (int)(t - c * DIM);
    int ic, jc, kc;
    ndec(gc, c, ic, jc, kc);
    const int fi = 2 * ic, fj = 2 * jc, fk = 2 * kc;
    const TA ti = (ic == 0 || ic == gc.nn[0] - 1) ? TA(1.0 / 1.5) : TA(0.5);
    const TA tj = (jc == 0 || jc == gc.nn[1] - 1) ? TA(1.0 / 1.5) : TA(0.5);
    TA tk = TA(1);
    if (DIM == 3) tk = (kc == 0 || kc == gc.nn[2] - 1) ? TA(1.0 / 1.5) : TA(0.5);
    constexpr int KR = DIM == 3 ? 1 : 0;
    TA acc = TA(0);
#pragma unroll
    for (int dj = -1; dj <= 1; dj++) {
        const int j = fj + dj;
        if (j < 0 || j >= gf.nn[1]) continue;
        TA accj = TA(0);
#pragma unroll
        for (int di = -1; di <= 1; di++) {
            const int i = fi + di;
            if (i < 0 || i >= gf.nn[0]) continue;
            TA acci = TA(0);
#pragma unroll
            for (int dk = -KR; dk <= KR; dk++) {
                const int k = fk + dk;
                if (DIM == 3 && (k < 0 || k >= gf.nn[2])) continue;
                const TA v = (TA)vf[nidx(gf, i, j, k) * DIM + d];
                acci += dk == 0 ? v : TA(0.5) * v;
            }
            accj += di == 0 ? acci : TA(0.5) * acci;
        }
        acc += dj == 0 ? accj : TA(0.5) * accj;
    }
    const TO bc = (TO)(acc * ti * tj * tk);
    vc[c * DIM + d] = bc;
    // first smoothing sweep of the coarse level from x = 0: x = omega * scale / diag * b
    if (j0.x) j0.x[c * DIM + d] = (TO)((*j0.omega) * j0.scale) * j0.dinv[c * DIM + d] * bc;
}

// One thread per fine node (all DIM components, contiguous loads of each parent): P =
// Phat diag(1/tw), the mean of the 1, 2, 4 or 8 parent values divided by their tw.  With an
// odd element count the last fine node along that axis has a single parent and takes its
// value (mgm.cu:198-244 averages over the parents that exist), so there P is not R^T.
template <int DIM, typename T>
__global__ void k_prolong(GridDev<DIM> gf, GridDev<DIM> gc, const T* __restrict__ vc, T* __restrict__ vf,
                          const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (skip && *skip) return;
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= gf.n_nodes) return;
    int i, j, k;
    ndec(gf, f, i, j, k);
    const int i0 = i >> 1, j0 = j >> 1, k0 = DIM == 3 ? k >> 1 : 0;
    // an odd fine node past the last coarse node (odd element count) has one parent
    const int i1 = min(i0 + (i & 1), gc.nn[0] - 1), j1 = min(j0 + (j & 1), gc.nn[1] - 1);
    const int k1 = DIM == 3 ? min(k0 + (k & 1), gc.nn[2] - 1) : 0;
    auto itw = [&](int c, int n) { return (c == 0 || c == n - 1) ? T(1.0 / 1.5) : T(0.5); };
    T acc[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) acc[d] = T(0);
    for (int cj = j0; cj <= j1; cj++) {
        const T wj = itw(cj, gc.nn[1]);
        for (int ci = i0; ci <= i1; ci++) {
            const T wij = wj * itw(ci, gc.nn[0]);
            for (int ck = k0; ck <= k1; ck++) {
                const T w = DIM == 3 ? wij * itw(ck, gc.nn[2]) : wij;
                const T* v = vc + nidx(gc, ci, cj, ck) * DIM;
#pragma unroll
                for (int d = 0; d < DIM; d++) acc[d] += w * v[d];
            }
        }
    }
    const int npar = (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1);  // the mean over the parents
    const T scale = npar == 1 ? T(1) : npar == 2 ? T(0.5) : npar == 4 ? T(0.25) : T(0.125);
#pragma unroll
    for (int d = 0; d < DIM; d++) vf[f * DIM + d] = acc[d] * scale;
}

// 3D prolongation by cells: one thread per coarse node (ic, jc, kc) writes the up-to-8 fine
// nodes (2ic + di, 2jc + dj, 2kc + dk), d in {0, 1}, from the up-to-8 coarse nodes
// (ic + a, jc + b, kc + c).  Each coarse value is read once per thread instead of once per
// fine child, and each thread writes two contiguous fine nodes (6 values) per (di, dj), so a
// warp's stores of consecutive kc are contiguous.  Per axis a fine node at 2c takes parent c,
// one at 2c + 1 the mean of c and c + 1, or c alone past the last coarse node (odd count):
// the same values as k_prolong.
template <typename T>
__global__ void __launch_bounds__(256) k_prolong_cells(GridDev<3> gf, GridDev<3> gc, const T* __restrict__ vc,
                                                       T* __restrict__ vf, const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (skip && *skip) return;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= gc.n_nodes) return;
    int ic, jc, kc;
    ndec(gc, c, ic, jc, kc);
    auto itw = [](int v, int n) { return (v == 0 || v == n - 1) ? T(1.0 / 1.5) : T(0.5); };
    const bool hx = ic + 1 < gc.nn[0], hy = jc + 1 < gc.nn[1], hz = kc + 1 < gc.nn[2];  // upper parents
    const bool fx = 2 * ic + 1 < gf.nn[0], fy = 2 * jc + 1 < gf.nn[1], fz = 2 * kc + 1 < gf.nn[2];  // odd children
    // z stage for the four (a, b) parent columns: values at fine k = 2kc (z0) and 2kc + 1 (z1)
    T z0[2][2][3], z1[2][2][3];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const bool ok = (a == 0 || hx) && (b == 0 || hy);
            const int pi = ic + (ok ? a : 0), pj = jc + (ok ? b : 0);
            const T wab = itw(pi, gc.nn[0]) * itw(pj, gc.nn[1]);
            const T* v0 = vc + nidx(gc, pi, pj, kc) * 3;
            const T w0 = wab * itw(kc, gc.nn[2]);
            T lo[3], hi[3];
#pragma unroll
            for (int d = 0; d < 3; d++) lo[d] = ok ? w0 * v0[d] : T(0);
            if (hz) {
                const T* v1 = vc + nidx(gc, pi, pj, kc + 1) * 3;
                const T w1 = wab * itw(kc + 1, gc.nn[2]);
#pragma unroll
                for (int d = 0; d < 3; d++) hi[d] = ok ? T(0.5) * (lo[d] + w1 * v1[d]) : T(0);
            } else {
#pragma unroll
                for (int d = 0; d < 3; d++) hi[d] = lo[d];
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                z0[a][b][d] = lo[d];
                z1[a][b][d] = hi[d];
            }
        }
    // y then x stages, written per (di, dj) as the two z-neighbouring fine nodes
#pragma unroll
    for (int di = 0; di < 2; di++) {
        if (di && !fx) continue;
#pragma unroll
        for (int dj = 0; dj < 2; dj++) {
            if (dj && !fy) continue;
            T o0[3], o1[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                // along y for column a, then along x
                T ya0[2], ya1[2];
#pragma unroll
                for (int a = 0; a < 2; a++) {
                    ya0[a] = dj == 0 ? z0[a][0][d] : (hy ? T(0.5) * (z0[a][0][d] + z0[a][1][d]) : z0[a][0][d]);
                    ya1[a] = dj == 0 ? z1[a][0][d] : (hy ? T(0.5) * (z1[a][0][d] + z1[a][1][d]) : z1[a][0][d]);
                }
                o0[d] = di == 0 ? ya0[0] : (hx ? T(0.5) * (ya0[0] + ya0[1]) : ya0[0]);
                o1[d] = di == 0 ? ya1[0] : (hx ? T(0.5) * (ya1[0] + ya1[1]) : ya1[0]);
            }
            T* out = vf + nidx(gf, 2 * ic + di, 2 * jc + dj, 2 * kc) * 3;
#pragma unroll
            for (int d = 0; d < 3; d++) out[d] = o0[d];
            if (fz) {
#pragma unroll
                for (int d = 0; d < 3; d++) out[3 + d] = o1[d];
            }
        }
    }
}

template <typename TI, typename TO>
int launch_restrict(const Grid& gf, const TI* vf, TO* vc, const int* skip, cudaStream_t st, Jacobi0<TO> j0) {
    const Grid gc = coarse_grid(gf);
    const unsigned nb = (unsigned)((gc.n_nodes * gf.dim + 255) / 256);
    pf::count_launch();
    if (gf.dim == 3)
        PF_CUDA(launch_pdl(k_restrict<3, TI, TO>, dim3(nb), dim3(256), 0, st, gdev<3>(gf), gdev<3>(gc), vf, vc, skip, j0));
    else
        PF_CUDA(launch_pdl(k_restrict<2, TI, TO>, dim3(nb), dim3(256), 0, st, gdev<2>(gf), gdev<2>(gc), vf, vc, skip, j0));
    PF_LAUNCH_CHECK("restrict launch");
    return PF_OK;
}
template <typename T>
int launch_prolong(const Grid& gf, const T* vc, T* vf, const int* skip, cudaStream_t st) {
    const Grid gc = coarse_grid(gf);
    const unsigned nb = (unsigned)((gf.n_nodes + 255) / 256);
    pf::count_launch();
    if (gf.dim == 3)
        PF_CUDA(launch_pdl(k_prolong_cells<T>, dim3((unsigned)((gc.n_nodes + 255) / 256)), dim3(256), 0, st,
                           gdev<3>(gf), gdev<3>(gc), vc, vf, skip));
    else
        PF_CUDA(launch_pdl(k_prolong<2, T>, dim3(nb), dim3(256), 0, st, gdev<2>(gf), gdev<2>(gc), vc, vf, skip));
    PF_LAUNCH_CHECK("prolong launch");
    return PF_OK;
}
template int launch_restrict<double, double>(const Grid&, const double*, double*, const int*, cudaStream_t,
                                            Jacobi0<double>);
template int launch_restrict<float, float>(const Grid&, const float*, float*, const int*, cudaStream_t,
                                          Jacobi0<float>);
template int launch_prolong<double>(const Grid&, const double*, double*, const int*, cudaStream_t);
template int launch_prolong<float>(const Grid&, const float*, float*, const int*, cudaStream_t);

// ---------------------------------------------------------------------------------------
// block-stencil matvec (levels >= 1): y_n = sum_o A[n,o] u_{n+o}
// A block covers 32 consecutive nodes; warp w gathers the neighbour offsets 3w..3w+2 for
// all 32 nodes (coalesced reads of the structure-of-arrays coefficients), the per-warp
// partial sums meet in shared memory and warp 0 adds them in a fixed order and applies the
// epilogue.  3D: 9 warps x 3 offsets, 2D: 3 warps x 3 offsets.
// HALF: A holds only the centre and the upper offsets o > c (c = NB/2 the centre, stored
// block q = o - c); a lower offset o < c uses the symmetry of the level operator,
// A[n, o] = A[n+o, -o]^T, i.e. block q = c - o of the neighbour n+o, transposed.  The
// neighbour's coefficients are read again by another block shortly after (from L2), so
// DRAM carries each coefficient once: (NB+1)/2 blocks per node instead of NB.  The half
// copy is tiled by 32 nodes, A[((n >> 5) * NH*BS + q*BS + a*DIM + b) * 32 + (n & 31)]:
// each tile's (NB+1)/2 * DIM^2 coefficient rows are one contiguous run (16 KB in 3D FP32),
// so DRAM streams through it instead of jumping between NH*BS planes of N values.
// ---------------------------------------------------------------------------------------
// Launch bounds: FP32 keeps 7 blocks per SM (32 registers); FP64 lets the compiler take 56
// registers (4 blocks per SM), measured faster than its default 40 for the FP64 solves.
template <int DIM, typename T, bool HALF>
__global__ void __launch_bounds__(DIM == 3 ? 288 : 96, (DIM == 3 && sizeof(T) == 4) ? 7 : 1)
    k_stencil_matvec(GridDev<DIM> g, const T* __restrict__ A, const T* __restrict__ u, Epi<T> epi) {
    pdl_wait();
    pdl_trigger();
    constexpr int NB = DIM == 3 ? 27 : 9, BS = DIM * DIM, NG = NB / 3, C = NB / 2;
    constexpr long long TS = (long long)(C + 1) * BS * 32;  // values per tile of the half copy
    __shared__ T s_part[NG][DIM][32];
    if (epi.skip && *epi.skip) return;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const long long n = (long long)blockIdx.x * 32 + l;
    const long long N = g.n_nodes;
    const bool valid = n < N;
    T acc[DIM];
#pragma unroll
    for (int a = 0; a < DIM; a++) acc[a] = T(0);
    if (valid) {
        int i, j, k;
        ndec(g, n, i, j, k);
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int o = 3 * w + q;
            const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = DIM == 3 ? o / 9 - 1 : 0;
            if (!nok(g, i + ox, j + oy, k + oz)) continue;
            const long long m = nidx(g, i + ox, j + oy, k + oz);
            T um[DIM];
#pragma unroll
            for (int b = 0; b < DIM; b++) um[b] = u[m * DIM + b];
            if (!HALF) {
#pragma unroll
                for (int a = 0; a < DIM; a++)
#pragma unroll
                    for (int b = 0; b < DIM; b++)
                        acc[a] = fma(A[((long long)(o * BS + a * DIM + b)) * N + n], um[b], acc[a]);
            } else if (o >= C) {
                const T* Aq = A + (n >> 5) * TS + (o - C) * BS * 32 + (n & 31);
#pragma unroll
                for (int a = 0; a < DIM; a++)
#pragma unroll
                    for (int b = 0; b < DIM; b++) acc[a] = fma(Aq[(a * DIM + b) * 32], um[b], acc[a]);
            } else {
                const T* Aq = A + (m >> 5) * TS + (C - o) * BS * 32 + (m & 31);
#pragma unroll
                for (int a = 0; a < DIM; a++)
#pragma unroll
                    for (int b = 0; b < DIM; b++) acc[a] = fma(Aq[(b * DIM + a) * 32], um[b], acc[a]);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < DIM; a++) s_part[w][a][l] = acc[a];
    __syncthreads();
    if (w != 0) return;
    double dot = 0.0;
    if (valid) {
        const T wgt = epi_omega(epi);
#pragma unroll
        for (int a = 0; a < DIM; a++) {
            T y = s_part[0][a][l];
#pragma unroll
            for (int v = 1; v < NG; v++) y += s_part[v][a][l];
            const long long gi = n * DIM + a;
            const T o = epi_apply(epi, gi, y, wgt);
            epi.out[gi] = o;
            if (epi.dot_partial) dot += (double)epi.dot_a[gi] * (double)(epi.dot_of_y ? y : o);
        }
    }
    if (epi.dot_partial) {
        dot = warp_sum(dot);
        if (l == 0) epi.dot_partial[blockIdx.x] = dot;
    }
}

template <typename T>
int launch_stencil_matvec(const Grid& g, const T* A, const T* u, const Epi<T>& epi, cudaStream_t st, bool half) {
    const unsigned nb = (unsigned)((g.n_nodes + 31) / 32);
    pf::count_launch();
    if (g.dim == 3) {
        if (half)
            PF_CUDA(launch_pdl(k_stencil_matvec<3, T, true>, dim3(nb), dim3(288), 0, st, gdev<3>(g), A, u, epi));
        else
            PF_CUDA(launch_pdl(k_stencil_matvec<3, T, false>, dim3(nb), dim3(288), 0, st, gdev<3>(g), A, u, epi));
    } else {
        if (half)
            PF_CUDA(launch_pdl(k_stencil_matvec<2, T, true>, dim3(nb), dim3(96), 0, st, gdev<2>(g), A, u, epi));
        else
            PF_CUDA(launch_pdl(k_stencil_matvec<2, T, false>, dim3(nb), dim3(96), 0, st, gdev<2>(g), A, u, epi));
    }
    PF_LAUNCH_CHECK("stencil matvec launch");
    return PF_OK;
}
long long stencil_matvec_num_blocks(const Grid& g) { return (g.n_nodes + 31) / 32; }
template int launch_stencil_matvec<double>(const Grid&, const double*, const double*, const Epi<double>&,
                                           cudaStream_t, bool);
template int launch_stencil_matvec<float>(const Grid&, const float*, const float*, const Epi<float>&, cudaStream_t,
                                          bool);

// half storage for the V-cycle: the centre and upper-offset blocks of the full FP64 stencil,
// converted to the V-cycle precision
template <typename T>
__global__ void k_stencil_half(long long N, int nh, int bs, int c, const double* __restrict__ A, T* __restrict__ H) {
    // tiles of 32 nodes (the last one zero-padded): H[(t * nh*bs + qab) * 32 + lane]
    const long long per_tile = (long long)nh * bs * 32;
    const long long total = ((N + 31) / 32) * per_tile;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long t = i / per_tile;
        const int r = (int)(i - t * per_tile), qab = r >> 5;
        const long long n = t * 32 + (r & 31);
        H[i] = n < N ? (T)A[(long long)(c * bs + qab) * N + n] : T(0);
    }
}
long long stencil_half_size(const Grid& g) {
    const int nb = g.dim == 3 ? 27 : 9;
    return ((g.n_nodes + 31) / 32) * 32 * ((nb + 1) / 2) * g.dof * g.dof;
}
template <typename T>
int launch_stencil_half(const Grid& g, const double* A, T* H, cudaStream_t st) {
    const int nb = g.dim == 3 ? 27 : 9, bs = g.dof * g.dof;
    const long long total = stencil_half_size(g);
    long long blocks = (total + 255) / 256;
    if (blocks > 8LL * kNumSM * 4) blocks = 8LL * kNumSM * 4;
    pf::count_launch();
    k_stencil_half<T><<<(unsigned)blocks, 256, 0, st>>>(g.n_nodes, (nb + 1) / 2, bs, nb / 2, A, H);
    PF_LAUNCH_CHECK("stencil half launch");
    return PF_OK;
}
template int launch_stencil_half<double>(const Grid&, const double*, double*, cudaStream_t);
template int launch_stencil_half<float>(const Grid&, const double*, float*, cudaStream_t);

// ---------------------------------------------------------------------------------------
// Galerkin level 1 from the element operator.
// With Phat_c the local interpolation from a coarse element's corners to its child c,
//   Phat^T (Z K Z) Phat = sum_C sum_c E_{C,c} (Z Phat_c)^T K0 (Z Phat_c)
// which for a coarse element C whose 3^DIM fine nodes carry no constraint is
// sum_c E_{C,c} Kc[c] with the fixed child matrices Kc[c] = Phat_c^T K0 Phat_c.  The
// identity rows of constrained DOFs add Phat^T (I - Z) Phat.  Each thread produces one
// dof x dof block (coarse node I, neighbour o) by gathering the coarse elements that
// contain I and I+o (owner computes, no atomics), then scales by 1/(tw_I tw_J).
// ---------------------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ int ccx(int l) {
    return kCXd(l);
}

// flags: per coarse element, 1 if any of its fine nodes has a constraint;
//        per coarse node, 1 if any fine node within distance 1 of 2I has a constraint.
template <int DIM>
__global__ void k_coarse_flags(GridDev<DIM> gf, GridDev<DIM> gc, const uint8_t* __restrict__ mask,
                               uint8_t* __restrict__ elem_flag, uint8_t* __restrict__ node_flag) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= gc.n_nodes) return;
    int ic, jc, kc;
    ndec(gc, c, ic, jc, kc);
    constexpr int KR = DIM == 3 ? 1 : 0;
    uint8_t nf = 0;
    for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
            for (int dk = -KR; dk <= KR; dk++) {
                const int fi = 2 * ic + di, fj = 2 * jc + dj, fk = 2 * kc + dk;
                if (nok(gf, fi, fj, fk) && mask[nidx(gf, fi, fj, fk)]) nf = 1;
            }
    node_flag[c] = nf;
    // coarse element with lower corner (ic, jc, kc)
    const bool has_elem = ic < gc.nel[0] && jc < gc.nel[1] && (DIM == 2 || kc < gc.nel[2]);
    if (has_elem) {
        uint8_t ef = 0;
        for (int di = 0; di <= 2; di++)
            for (int dj = 0; dj <= 2; dj++)
                for (int dk = 0; dk <= 2 * KR; dk++)
                    if (mask[nidx(gf, 2 * ic + di, 2 * jc + dj, 2 * kc + dk)]) ef = 1;
        const long long e = DIM == 3 ? ((long long)ic * gc.nel[1] + jc) * gc.nel[2] + kc : (long long)ic * gc.nel[1] + jc;
        elem_flag[e] = ef;
    }
}

template <int DIM>
__global__ void __launch_bounds__(128) k_galerkin_l0(GridDev<DIM> gf, GridDev<DIM> gc, const double* __restrict__ E,
                                                      const uint8_t* __restrict__ mask,
                                                      const uint8_t* __restrict__ elem_flag,
                                                      const uint8_t* __restrict__ node_flag,
                                                      const double* __restrict__ K0,  // (NC*DIM)^2
                                                      const double* __restrict__ Kc,  // NC x (NC*DIM)^2
                                                      double* __restrict__ A) {
    constexpr int NC = DIM == 3 ? 8 : 4, ND = NC * DIM, NB = DIM == 3 ? 27 : 9, BS = DIM * DIM;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long Nc = gc.n_nodes;
    if (tid >= Nc * NB) return;
    const int o = (int)(tid / Nc);
    const long long I = tid - (long long)o * Nc;
    int ic, jc, kc;
    ndec(gc, I, ic, jc, kc);
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = DIM == 3 ? o / 9 - 1 : 0;
    double blk[BS];
#pragma unroll
    for (int a = 0; a < BS; a++) blk[a] = 0.0;
    const int ti = ic + ox, tj = jc + oy, tk = kc + oz;
    if (nok(gc, ti, tj, tk)) {
        // coarse elements containing I as local corner LI
        for (int LI = 0; LI < NC; LI++) {
            const int ex = ic - kCXd(LI), ey = jc - kCYd(LI), ez = DIM == 3 ? kc - kCZd(LI) : 0;
            // past the last coarse node of an axis with an odd element count lies a virtual
            // coarse element: its far corners do not exist and only its near children do
            const bool vx = ex == gc.nel[0] && gf.nel[0] > 2 * gc.nel[0];
            const bool vy = ey == gc.nel[1] && gf.nel[1] > 2 * gc.nel[1];
            const bool vz = DIM == 3 && ez == gc.nel[2] && gf.nel[2] > 2 * gc.nel[2];
            if (ex < 0 || ey < 0 || (ex >= gc.nel[0] && !vx) || (ey >= gc.nel[1] && !vy)) continue;
            if (DIM == 3 && (ez < 0 || (ez >= gc.nel[2] && !vz))) continue;
            // J must be a corner of the same element
            const int lx = kCXd(LI) + ox, ly = kCYd(LI) + oy, lz = DIM == 3 ? kCZd(LI) + oz : 0;
            if (lx < 0 || lx > 1 || ly < 0 || ly > 1 || lz < 0 || lz > 1) continue;
            if ((vx && (kCXd(LI) || lx)) || (vy && (kCYd(LI) || ly)) || (vz && (kCZd(LI) || lz))) continue;
            int LJ = 0;
            for (int q = 0; q < NC; q++)
                if (kCXd(q) == lx && kCYd(q) == ly && (DIM == 2 || kCZd(q) == lz)) LJ = q;
            const bool virt = vx || vy || vz;
            const long long ce = DIM == 3 ? ((long long)ex * gc.nel[1] + ey) * gc.nel[2] + ez : (long long)ex * gc.nel[1] + ey;
            const bool dirty = virt || elem_flag[ce] != 0;  // virtual elements check their masks
            for (int c = 0; c < NC; c++) {
                const int fx = 2 * ex + kCXd(c), fy = 2 * ey + kCYd(c), fz = DIM == 3 ? 2 * ez + kCZd(c) : 0;
                if (fx >= gf.nel[0] || fy >= gf.nel[1] || (DIM == 3 && fz >= gf.nel[2])) continue;
                const long long fe = DIM == 3 ? ((long long)fx * gf.nel[1] + fy) * gf.nel[2] + fz : (long long)fx * gf.nel[1] + fy;
                const double we = E[fe];
                if (!dirty) {
                    const double* kc_ = Kc + (long long)c * ND * ND;
#pragma unroll
                    for (int a = 0; a < DIM; a++)
#pragma unroll
                        for (int b = 0; b < DIM; b++) blk[a * DIM + b] += we * __ldg(kc_ + (LI * DIM + a) * ND + LJ * DIM + b);
                } else {
                    // masked child: sum_{l,l2} Phat_c[l][LI] z(l,a) K0[(l,a),(l2,b)] z(l2,b) Phat_c[l2][LJ]
                    for (int l = 0; l < NC; l++) {
                        const int nxl = kCXd(c) + kCXd(l), nyl = kCYd(c) + kCYd(l), nzl = DIM == 3 ? kCZd(c) + kCZd(l) : 0;
                        double pl = (1.0 - 0.5 * abs(nxl - 2 * kCXd(LI))) * (1.0 - 0.5 * abs(nyl - 2 * kCYd(LI)));
                        if (DIM == 3) pl *= 1.0 - 0.5 * abs(nzl - 2 * kCZd(LI));
                        if (pl == 0.0) continue;
                        const uint8_t ml = mask ? mask[nidx(gf, 2 * ex + nxl, 2 * ey + nyl, 2 * ez + nzl)] : 0;
                        for (int l2 = 0; l2 < NC; l2++) {
                            const int nx2 = kCXd(c) + kCXd(l2), ny2 = kCYd(c) + kCYd(l2), nz2 = DIM == 3 ? kCZd(c) + kCZd(l2) : 0;
                            double p2 = (1.0 - 0.5 * abs(nx2 - 2 * kCXd(LJ))) * (1.0 - 0.5 * abs(ny2 - 2 * kCYd(LJ)));
                            if (DIM == 3) p2 *= 1.0 - 0.5 * abs(nz2 - 2 * kCZd(LJ));
                            if (p2 == 0.0) continue;
                            const uint8_t m2 = mask ? mask[nidx(gf, 2 * ex + nx2, 2 * ey + ny2, 2 * ez + nz2)] : 0;
                            const double f = we * pl * p2;
                            for (int a = 0; a < DIM; a++) {
                                if (ml & (1 << a)) continue;
                                for (int b = 0; b < DIM; b++) {
                                    if (m2 & (1 << b)) continue;
                                    blk[a * DIM + b] += f * K0[(l * DIM + a) * ND + l2 * DIM + b];
                                }
                            }
                        }
                    }
                }
            }
        }
        // identity rows of constrained fine DOFs: sum_n Phat[n,I] Phat[n,J] on the diagonal
        if (node_flag[I]) {
            constexpr int KR = DIM == 3 ? 1 : 0;
            for (int di = -1; di <= 1; di++)
                for (int dj = -1; dj <= 1; dj++)
                    for (int dk = -KR; dk <= KR; dk++) {
                        const int fi = 2 * ic + di, fj = 2 * jc + dj, fk = 2 * kc + dk;
                        if (!nok(gf, fi, fj, fk)) continue;
                        const int ei = fi - 2 * ti, ej = fj - 2 * tj, ek = fk - 2 * tk;
                        if (ei < -1 || ei > 1 || ej < -1 || ej > 1 || ek < -1 || ek > 1) continue;
                        const uint8_t m = mask[nidx(gf, fi, fj, fk)];
                        if (!m) continue;
                        const double w = half_pow((di != 0) + (dj != 0) + (dk != 0)) *
                                         half_pow((ei != 0) + (ej != 0) + (ek != 0));
                        for (int a = 0; a < DIM; a++)
                            if (m & (1 << a)) blk[a * DIM + a] += w;
                    }
        }
        const double s = 1.0 / (total_weight(gc, ic, jc, kc) * total_weight(gc, ti, tj, tk));
#pragma unroll
        for (int a = 0; a < BS; a++) blk[a] *= s;
    }
#pragma unroll
    for (int a = 0; a < BS; a++) A[((long long)(o * BS + a)) * Nc + I] = blk[a];
}

// child matrices Kc[c] = Phat_c^T K0 Phat_c (host)
void galerkin_child_matrices(int dim, const double* K0, double* Kc) {
    const int NC = dim == 3 ? 8 : 4, ND = NC * dim;
    for (int c = 0; c < NC; c++) {
        double P[8][8];  // P[l][L]: weight of coarse corner L at child corner l
        for (int l = 0; l < NC; l++)
            for (int L = 0; L < NC; L++) {
                const int fx = kCXd(c) + kCXd(l), fy = kCYd(c) + kCYd(l), fz = dim == 3 ? kCZd(c) + kCZd(l) : 0;
                double w = (1.0 - 0.5 * abs(fx - 2 * kCXd(L))) * (1.0 - 0.5 * abs(fy - 2 * kCYd(L)));
                if (dim == 3) w *= 1.0 - 0.5 * abs(fz - 2 * kCZd(L));
                P[l][L] = w;
            }
        double* out = Kc + (long long)c * ND * ND;
        for (int L = 0; L < NC; L++)
            for (int a = 0; a < dim; a++)
                for (int L2 = 0; L2 < NC; L2++)
                    for (int b = 0; b < dim; b++) {
                        double s = 0.0;
                        for (int l = 0; l < NC; l++) {
                            if (P[l][L] == 0.0) continue;
                            for (int l2 = 0; l2 < NC; l2++) {
                                if (P[l2][L2] == 0.0) continue;
                                s += P[l][L] * K0[(l * dim + a) * ND + l2 * dim + b] * P[l2][L2];
                            }
                        }
                        out[(L * dim + a) * ND + L2 * dim + b] = s;
                    }
    }
}

int launch_coarse_flags(const Grid& gf, const uint8_t* mask, uint8_t* elem_flag, uint8_t* node_flag, cudaStream_t st) {
    const Grid gc = coarse_grid(gf);
    const unsigned nb = (unsigned)((gc.n_nodes + 255) / 256);
    pf::count_launch();
    if (gf.dim == 3)
        k_coarse_flags<3><<<nb, 256, 0, st>>>(gdev<3>(gf), gdev<3>(gc), mask, elem_flag, node_flag);
    else
        k_coarse_flags<2><<<nb, 256, 0, st>>>(gdev<2>(gf), gdev<2>(gc), mask, elem_flag, node_flag);
    PF_LAUNCH_CHECK("coarse flags launch");
    return PF_OK;
}

int launch_galerkin_l0(const Grid& gf, const double* E, const uint8_t* mask, const uint8_t* elem_flag,
                       const uint8_t* node_flag, const double* K0_dev, const double* Kc_dev, double* A, cudaStream_t st) {
    const Grid gc = coarse_grid(gf);
    const int NB = gf.dim == 3 ? 27 : 9;
    const long long n = gc.n_nodes * NB;
    const unsigned nb = (unsigned)((n + 127) / 128);
    pf::count_launch();
    if (gf.dim == 3)
        k_galerkin_l0<3><<<nb, 128, 0, st>>>(gdev<3>(gf), gdev<3>(gc), E, mask, elem_flag, node_flag, K0_dev, Kc_dev, A);
    else
        k_galerkin_l0<2><<<nb, 128, 0, st>>>(gdev<2>(gf), gdev<2>(gc), E, mask, elem_flag, node_flag, K0_dev, Kc_dev, A);
    PF_LAUNCH_CHECK("galerkin l0 launch");
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// Galerkin level l+1 from the level-l block stencil:
//   A_c[I,J] = sum_{n in supp I} sum_{m in supp J, |m-n|<=1} Phat[n,I] A[n, m-n] Phat[m,J] / (tw_I tw_J)
// Per axis, the admissible (dn, dm) offset pairs depend only on the neighbour offset o.
// ---------------------------------------------------------------------------------------
__constant__ int c_pairs[3][7][2];  // [o+1][pair][dn, dm]
__constant__ int c_npairs[3];

template <int DIM>
__global__ void __launch_bounds__(128) k_galerkin_l1p(GridDev<DIM> gf, GridDev<DIM> gc, const double* __restrict__ Af,
                                                       double* __restrict__ Ac) {
    constexpr int NB = DIM == 3 ? 27 : 9, BS = DIM * DIM;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long Nc = gc.n_nodes, Nf = gf.n_nodes;
    if (tid >= Nc * NB) return;
    const int o = (int)(tid / Nc);
    const long long I = tid - (long long)o * Nc;
    int ic, jc, kc;
    ndec(gc, I, ic, jc, kc);
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = DIM == 3 ? o / 9 - 1 : 0;
    double blk[BS];
#pragma unroll
    for (int a = 0; a < BS; a++) blk[a] = 0.0;
    const int ti = ic + ox, tj = jc + oy, tk = kc + oz;
    if (nok(gc, ti, tj, tk)) {
        const int npx = c_npairs[ox + 1], npy = c_npairs[oy + 1], npz = DIM == 3 ? c_npairs[oz + 1] : 1;
        for (int px = 0; px < npx; px++) {
            const int dnx = c_pairs[ox + 1][px][0], dmx = c_pairs[ox + 1][px][1];
            const int nx_ = 2 * ic + dnx, mx = 2 * ti + dmx;
            if (nx_ < 0 || nx_ >= gf.nn[0] || mx < 0 || mx >= gf.nn[0]) continue;
            for (int py = 0; py < npy; py++) {
                const int dny = c_pairs[oy + 1][py][0], dmy = c_pairs[oy + 1][py][1];
                const int ny_ = 2 * jc + dny, my = 2 * tj + dmy;
                if (ny_ < 0 || ny_ >= gf.nn[1] || my < 0 || my >= gf.nn[1]) continue;
                for (int pz = 0; pz < npz; pz++) {
                    int dnz = 0, dmz = 0, nz_ = 0, mz = 0;
                    if (DIM == 3) {
                        dnz = c_pairs[oz + 1][pz][0];
                        dmz = c_pairs[oz + 1][pz][1];
                        nz_ = 2 * kc + dnz;
                        mz = 2 * tk + dmz;
                        if (nz_ < 0 || nz_ >= gf.nn[2] || mz < 0 || mz >= gf.nn[2]) continue;
                    }
                    const double w = half_pow((dnx != 0) + (dny != 0) + (dnz != 0)) *
                                     half_pow((dmx != 0) + (dmy != 0) + (dmz != 0));
                    const long long n = nidx(gf, nx_, ny_, nz_);
                    const int rx = mx - nx_, ry = my - ny_, rz = DIM == 3 ? mz - nz_ : 0;
                    const int on = (rx + 1) + 3 * (ry + 1) + (DIM == 3 ? 9 * (rz + 1) : 0);
#pragma unroll
                    for (int a = 0; a < BS; a++) blk[a] += w * Af[((long long)(on * BS + a)) * Nf + n];
                }
            }
        }
        const double s = 1.0 / (total_weight(gc, ic, jc, kc) * total_weight(gc, ti, tj, tk));
#pragma unroll
        for (int a = 0; a < BS; a++) blk[a] *= s;
    }
#pragma unroll
    for (int a = 0; a < BS; a++) Ac[((long long)(o * BS + a)) * Nc + I] = blk[a];
}

// One axis of the Galerkin product of a 3D level >= 2.  R = D Phat^T and P = Phat D are
// tensor products of per-axis factors (linear-interpolation weights 0.5^|d|, the per-axis
// part 1/1.5 or 1/2 of 1/tw, the bounds of each axis), so A_c = R A P is three one-axis
// products, x, then y, then z, each on a grid coarsened along the axes already done.  An
// output entry (node I, offset O) sums over the admissible (dn, dm) pairs of its axis only
// (at most 7, against up to 343 triples in k_galerkin_l1p): 2197 instead of 5 x 13^3 terms per
// coarse node summed over its 27 offsets, with the first pass on the fine grid coalesced.  Same
// operator, other rounding order.
template <int AX>
__global__ void __launch_bounds__(128) k_galerkin_axis(GridDev<3> gi, GridDev<3> go, const double* __restrict__ Si,
                                                       double* __restrict__ So) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long No = go.n_nodes, Ni = gi.n_nodes;
    if (tid >= No * 27) return;
    const int o = (int)(tid / No);
    const long long I = tid - (long long)o * No;
    int c[3];
    ndec(go, I, c[0], c[1], c[2]);
    const int oo[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
    const int Ia = c[AX], Ta = Ia + oo[AX];
    double blk[9];
#pragma unroll
    for (int a = 0; a < 9; a++) blk[a] = 0.0;
    if (Ta >= 0 && Ta < go.nn[AX]) {
        const int np = c_npairs[oo[AX] + 1];
        for (int p = 0; p < np; p++) {
            const int dn = c_pairs[oo[AX] + 1][p][0], dm = c_pairs[oo[AX] + 1][p][1];
            const int na = 2 * Ia + dn, ma = 2 * Ta + dm;
            if (na < 0 || na >= gi.nn[AX] || ma < 0 || ma >= gi.nn[AX]) continue;
            const double w = (dn != 0 ? 0.5 : 1.0) * (dm != 0 ? 0.5 : 1.0);
            int ci[3] = {c[0], c[1], c[2]}, ri[3] = {oo[0], oo[1], oo[2]};
            ci[AX] = na;
            ri[AX] = ma - na;
            const long long n = nidx(gi, ci[0], ci[1], ci[2]);
            const int on = (ri[0] + 1) + 3 * (ri[1] + 1) + 9 * (ri[2] + 1);
#pragma unroll
            for (int a = 0; a < 9; a++) blk[a] += w * Si[((long long)(on * 9 + a)) * Ni + n];
        }
        const int nn = go.nn[AX];
        const double s = 1.0 / (((Ia == 0 || Ia == nn - 1) ? 1.5 : 2.0) * ((Ta == 0 || Ta == nn - 1) ? 1.5 : 2.0));
#pragma unroll
        for (int a = 0; a < 9; a++) blk[a] *= s;
    }
#pragma unroll
    for (int a = 0; a < 9; a++) So[((long long)(o * 9 + a)) * No + I] = blk[a];
}

static bool g_pairs_ready = false;
static int init_pairs() {
    if (g_pairs_ready) return PF_OK;
    int pairs[3][7][2] = {};
    int np[3] = {0, 0, 0};
    for (int o = -1; o <= 1; o++)
        for (int dn = -1; dn <= 1; dn++)
            for (int dm = -1; dm <= 1; dm++) {
                const int r = 2 * o + dm - dn;
                if (r < -1 || r > 1) continue;
                pairs[o + 1][np[o + 1]][0] = dn;
                pairs[o + 1][np[o + 1]][1] = dm;
                np[o + 1]++;
            }
    PF_CUDA(cudaMemcpyToSymbol(c_pairs, pairs, sizeof(pairs)));
    PF_CUDA(cudaMemcpyToSymbol(c_npairs, np, sizeof(np)));
    g_pairs_ready = true;
    return PF_OK;
}

int launch_galerkin_l1p(const Grid& gf, const double* Af, double* Ac, cudaStream_t st) {
    int s = init_pairs();
    if (s) return s;
    const Grid gc = coarse_grid(gf);
    const int NB = gf.dim == 3 ? 27 : 9;
    const unsigned nb = (unsigned)((gc.n_nodes * NB + 127) / 128);
    pf::count_launch();
    if (gf.dim == 3)
        k_galerkin_l1p<3><<<nb, 128, 0, st>>>(gdev<3>(gf), gdev<3>(gc), Af, Ac);
    else
        k_galerkin_l1p<2><<<nb, 128, 0, st>>>(gdev<2>(gf), gdev<2>(gc), Af, Ac);
    PF_LAUNCH_CHECK("galerkin l1p launch");
    return PF_OK;
}

// the fine grid with one axis coarsened (element count halved, floored)
static Grid coarsen_axis(const Grid& g, int ax) {
    int nel[3] = {g.nel[0], g.nel[1], g.nel[2]};
    nel[ax] /= 2;
    return make_grid(g.dim, nel);
}

long long galerkin_sep_scratch(const Grid& gf) {
    if (gf.dim != 3) return 0;
    const Grid g1 = coarsen_axis(gf, 0), g2 = coarsen_axis(g1, 1);
    return 243LL * (g1.n_nodes + g2.n_nodes);
}

int launch_galerkin_sep(const Grid& gf, const double* Af, double* Ac, double* scratch, cudaStream_t st) {
    if (gf.dim != 3) return launch_galerkin_l1p(gf, Af, Ac, st);
    int s = init_pairs();
    if (s) return s;
    const Grid g1 = coarsen_axis(gf, 0), g2 = coarsen_axis(g1, 1), gc = coarsen_axis(g2, 2);
    double* S1 = scratch;
    double* S2 = scratch + 243LL * g1.n_nodes;
    auto nb = [](const Grid& g) { return (unsigned)((g.n_nodes * 27 + 127) / 128); };
    pf::count_launch(3);
    k_galerkin_axis<0><<<nb(g1), 128, 0, st>>>(gdev<3>(gf), gdev<3>(g1), Af, S1);
    k_galerkin_axis<1><<<nb(g2), 128, 0, st>>>(gdev<3>(g1), gdev<3>(g2), S1, S2);
    k_galerkin_axis<2><<<nb(gc), 128, 0, st>>>(gdev<3>(g2), gdev<3>(gc), S2, Ac);
    PF_LAUNCH_CHECK("separable galerkin launch");
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// stencil diagonal -> inverse diagonal, precision conversion, dense export
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_stencil_dinv(long long N, int dim, const double* __restrict__ A, T* __restrict__ dinv) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * dim) return;
    const long long n = t / dim;
    const int a = (int)(t - n * dim);
    const int oc = dim == 3 ? 13 : 4, BS = dim * dim;
    dinv[t] = (T)(1.0 / A[((long long)(oc * BS + a * dim + a)) * N + n]);
}

template <typename T>
int launch_stencil_dinv(const Grid& g, const double* A, T* dinv, cudaStream_t st) {
    const long long n = g.n_nodes * g.dim;
    pf::count_launch();
    k_stencil_dinv<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g.n_nodes, g.dim, A, dinv);
    PF_LAUNCH_CHECK("stencil dinv launch");
    return PF_OK;
}
template int launch_stencil_dinv<double>(const Grid&, const double*, double*, cudaStream_t);
template int launch_stencil_dinv<float>(const Grid&, const double*, float*, cudaStream_t);

template <int DIM>
__global__ void k_stencil_to_dense(GridDev<DIM> g, const double* __restrict__ A, double* __restrict__ M, long long ld) {
    constexpr int NB = DIM == 3 ? 27 : 9, BS = DIM * DIM;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long N = g.n_nodes;
    if (t >= N * NB * BS) return;
    const long long n = t % N;
    const int ob = (int)(t / N);
    const int o = ob / BS, ab = ob % BS, a = ab / DIM, b = ab % DIM;
    int i, j, k;
    ndec(g, n, i, j, k);
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = DIM == 3 ? o / 9 - 1 : 0;
    if (!nok(g, i + ox, j + oy, k + oz)) return;
    const long long m = nidx(g, i + ox, j + oy, k + oz);
    M[(n * DIM + a) * ld + m * DIM + b] = A[t];
}

int launch_stencil_to_dense(const Grid& g, const double* A, double* M, long long ld, cudaStream_t st) {
    const int NB = g.dim == 3 ? 27 : 9;
    const long long n = g.n_nodes * NB * g.dim * g.dim;
    pf::count_launch();
    if (g.dim == 3)
        k_stencil_to_dense<3><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(gdev<3>(g), A, M, ld);
    else
        k_stencil_to_dense<2><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(gdev<2>(g), A, M, ld);
    PF_LAUNCH_CHECK("stencil to dense launch");
    return PF_OK;
}

__global__ void k_d2f(long long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
int launch_d2f(long long n, const double* a, float* b, cudaStream_t st) {
    long long nb = (n + 255) / 256;
    if (nb > 4 * kNumSM * 8) nb = 4 * kNumSM * 8;
    if (nb < 1) nb = 1;
    pf::count_launch();
    k_d2f<<<(unsigned)nb, 256, 0, st>>>(n, a, b);
    PF_LAUNCH_CHECK("d2f launch");
    return PF_OK;
}

__global__ void k_d2bf(long long n, const double* __restrict__ a, __nv_bfloat16* __restrict__ b) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = __double2bfloat16(a[i]);
}
int launch_d2bf(long long n, const double* a, __nv_bfloat16* b, cudaStream_t st) {
    long long nb = (n + 255) / 256;
    if (nb > 4 * kNumSM * 8) nb = 4 * kNumSM * 8;
    if (nb < 1) nb = 1;
    pf::count_launch();
    k_d2bf<<<(unsigned)nb, 256, 0, st>>>(n, a, b);
    PF_LAUNCH_CHECK("d2bf launch");
    return PF_OK;
}

}  // namespace pf
