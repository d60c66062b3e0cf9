// Level-1 coarse operator applied element by element (no assembled coefficients).
//
// With trilinear interpolation Phat and the reference's normalised transfers
// R = D Phat^T, P = Phat D, D = diag(1/tw) (pyFANTOM/core/CUDA/Kernels/mgm.cu:1-244), the
// level-1 Galerkin operator is A1 = R (Z K Z + I - Z) P = D A^ D with
//   A^ = sum over coarse elements C of M_C,
//   M_C = sum_c E_{C,c} Kc[c],  Kc[c] = Phat_c^T K0 Phat_c   (C touches no constraint),
// where c runs over the 8 children of C.  Child c is child 0 reflected along the axes of
// its bits, and K0 of a box element is invariant under those reflections, so in the Walsh
// basis of C's corners (v = T u, the basis the fine matvec uses, T K0 T^T / 64 block
// diagonal)
//   T M_C T^T / 64 = B0 o Ehat[p(i) ^ p(j)],   Ehat_k = sum_c E_{C,c} (-1)^{popcount(c & k)},
// with B0 = T Kc[0] T^T / 64 and p(i) the reflection-parity class of Walsh slot i (mode m,
// component a: p = m ^ (1 << a)).  For isotropic box elements B0 has 279 nonzeros (150
// distinct by symmetry) in a fixed pattern, and the rows of the rigid translations (mode 0)
// vanish: one coarse element costs 279 + 150 multiply-adds on 8 precomputed Ehat values
// and no coefficient traffic, where the assembled stencil streams 126 coefficients per
// coarse node.
//
// Coarse elements with a constrained fine node ("dirty": their Z-masked children) keep an
// explicit Walsh-basis matrix: every coefficient pair (I, J) of the dirty part of A^ (the
// masked children of all dirty elements containing I and J) is assigned to the first dirty
// element (in element order) that contains both I and J, so the dirty matrices sum to
// exactly that part.  A dirty element is marked by Ehat_0 = -(index + 1) (Ehat_0 = sum E > 0
// otherwise), confirmed against the dirty list.  The identity rows Phat^T (I - Z) Phat are
// applied per coarse node in the physical basis (27 neighbours per component) by the owner
// of the node: inside a Walsh-basis matrix their O(1) entries would be mixed with the
// O(E_min) stiffness of void children, which FP32 cannot resolve (SIMP densities reach
// 1e-9 of the solid at a clamped face).
//
// The matvec is an x-march like the fine one (csrc/elemop.cu): warps cover element rows in
// y, lanes element columns in z, the element's Walsh transform is formed from the two
// faces, D is applied to u on load and to y at the owner, rows are exchanged through
// shared memory once per step; owner computes, no atomics, fixed summation order.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "coarse.cuh"
#include "common.cuh"
#include "elemop.cuh"
#include "mgkern.cuh"

namespace pf {

// coefficient index (0..149) of Walsh entry (i, j), i = m*3 + a, or -1 for a structural zero
// of B0 for isotropic box elements (rows and columns 0..2 are the rigid translations)
__host__ __device__ constexpr int coarse_pat(int i, int j) {
    constexpr int t[24][24] = {
        {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {-1, -1, -1, 0, -1, -1, -1, 1, -1, 2, 3, -1, -1, -1, 4, 5, -1, 6, -1, 7, 8, 9, 10, 11},
        {-1, -1, -1, -1, 12, -1, 13, -1, -1, 14, 15, -1, -1, -1, -1, -1, 16, -1, 17, -1, -1, 18, 19, -1},
        {-1, -1, -1, -1, -1, 20, -1, -1, -1, -1, -1, 21, 22, -1, -1, 23, -1, 24, 25, -1, -1, 26, -1, 27},
        {-1, -1, -1, -1, 13, -1, 28, -1, -1, 29, 30, -1, -1, -1, -1, -1, 31, -1, 32, -1, -1, 33, 34, -1},
        {-1, -1, -1, 1, -1, -1, -1, 35, -1, 36, 37, -1, -1, -1, 38, 39, -1, 40, -1, 41, 42, 43, 44, 45},
        {-1, -1, -1, -1, -1, -1, -1, -1, 46, -1, -1, 47, -1, 48, -1, -1, 49, -1, -1, 50, 51, -1, 52, 53},
        {-1, -1, -1, 2, 14, -1, 29, 36, -1, 54, 55, -1, -1, -1, 56, 57, 58, 59, 60, 61, 62, 63, 64, 65},
        {-1, -1, -1, 3, 15, -1, 30, 37, -1, 55, 66, -1, -1, -1, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76},
        {-1, -1, -1, -1, -1, 21, -1, -1, 47, -1, -1, 77, 78, 79, -1, 80, 81, 82, 83, 84, 85, 86, 87, 88},
        {-1, -1, -1, -1, -1, 22, -1, -1, -1, -1, -1, 78, 89, -1, -1, 90, -1, 91, 92, -1, -1, 93, -1, 94},
        {-1, -1, -1, -1, -1, -1, -1, -1, 48, -1, -1, 79, -1, 95, -1, -1, 96, -1, -1, 97, 98, -1, 99, 100},
        {-1, -1, -1, 4, -1, -1, -1, 38, -1, 56, 67, -1, -1, -1, 101, 102, -1, 103, -1, 104, 105, 106, 107, 108},
        {-1, -1, -1, 5, -1, 23, -1, 39, -1, 57, 68, 80, 90, -1, 102, 109, -1, 110, 111, 112, 113, 114, 115, 116},
        {-1, -1, -1, -1, 16, -1, 31, -1, 49, 58, 69, 81, -1, 96, -1, -1, 117, -1, 118, 119, 120, 121, 122, 123},
        {-1, -1, -1, 6, -1, 24, -1, 40, -1, 59, 70, 82, 91, -1, 103, 110, -1, 124, 125, 126, 127, 128, 129, 130},
        {-1, -1, -1, -1, 17, 25, 32, -1, -1, 60, 71, 83, 92, -1, -1, 111, 118, 125, 131, -1, -1, 132, 133, 134},
        {-1, -1, -1, 7, -1, -1, -1, 41, 50, 61, 72, 84, -1, 97, 104, 112, 119, 126, -1, 135, 136, 137, 138, 139},
        {-1, -1, -1, 8, -1, -1, -1, 42, 51, 62, 73, 85, -1, 98, 105, 113, 120, 127, -1, 136, 140, 141, 142, 143},
        {-1, -1, -1, 9, 18, 26, 33, 43, -1, 63, 74, 86, 93, -1, 106, 114, 121, 128, 132, 137, 141, 144, 145, 146},
        {-1, -1, -1, 10, 19, -1, 34, 44, 52, 64, 75, 87, -1, 99, 107, 115, 122, 129, 133, 138, 142, 145, 147, 148},
        {-1, -1, -1, 11, -1, 27, -1, 45, 53, 65, 76, 88, 94, 100, 108, 116, 123, 130, 134, 139, 143, 146, 148, 149},
    };
    return t[i][j];
}
constexpr int kCoarseCoefs = 150;
// reflection-parity class of Walsh slot i = m*3 + a
__host__ __device__ constexpr int wclass(int i) { return (i / 3) ^ (1 << (i % 3)); }
// Walsh slot of component a in class q
__host__ __device__ constexpr int wslot(int q, int a) { return (q ^ (1 << a)) * 3 + a; }

template <typename T>
struct CoarseCoef {
    T b[kCoarseCoefs];
};

// compile-time unrolled loop: f(std::integral_constant<int, 0>) ... f(<N-1>)
template <int N>
struct Unroll {
    template <typename F>
    __device__ __forceinline__ static void run(F&& f) {
        Unroll<N - 1>::run(f);
        f(std::integral_constant<int, N - 1>{});
    }
};
template <>
struct Unroll<0> {
    template <typename F>
    __device__ __forceinline__ static void run(F&&) {}
};

static int host_walsh(int m, int l) {
    const int pos[3] = {kCXd(l), kCYd(l), kCZd(l)};
    int s = 1;
    for (int a = 0; a < 3; a++)
        if ((m >> a) & 1) s *= pos[a] ? 1 : -1;
    return s;
}

// B0 = T Kc[0] T^T / 64 checked against the pattern; PF_UNSUPPORTED if K0 does not have it
int coarse_factorise(const Op* op, double* coef /* [150] */) {
    if (op->grid.dim != 3) return fail(PF_UNSUPPORTED, "element-level coarse operator: 3D only");
    std::vector<double> Kc(8 * 24 * 24);
    galerkin_child_matrices(3, op->K0, Kc.data());
    const double* K = Kc.data();  // child 0 (lowest corner)
    double B[24][24], tmp[24][24];
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            double s = 0.0;
            for (int l = 0; l < 8; l++) s += host_walsh(i / 3, l) * K[(l * 3 + i % 3) * 24 + j];
            tmp[i][j] = s;
        }
    double bmax = 0.0;
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            double s = 0.0;
            for (int l = 0; l < 8; l++) s += tmp[i][l * 3 + j % 3] * host_walsh(j / 3, l);
            B[i][j] = s / 64.0;
            bmax = fmax(bmax, fabs(B[i][j]));
        }
    const double tol = 1e-12 * bmax;
    for (int q = 0; q < kCoarseCoefs; q++) coef[q] = 0.0;
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) {
            const int q = coarse_pat(i, j);
            if (q < 0) {
                if (fabs(B[i][j]) > tol)
                    return fail(PF_UNSUPPORTED, "coarse operator: K0 lacks the isotropic-box structure (%d,%d)", i, j);
            } else {
                if (fabs(B[i][j] - B[j][i]) > tol) return fail(PF_UNSUPPORTED, "coarse operator: B0 not symmetric");
                coef[q] = B[i][j];
            }
        }
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// setup: dirty-element list, Ehat, dirty Walsh matrices
// ---------------------------------------------------------------------------------------
constexpr int kScanThreads = 1024;  // flags per block of the compaction

// Stream compaction of a flag array in index order, in two passes: block b counts the
// flags of items [1024 b, 1024 (b + 1)); then every block adds the counts of the blocks
// before it and places its items with a ballot scan.  map[i] = rank of item i among the
// flagged items (or -1), list[rank] = i (rank < cap), *count = number of flagged items.
__global__ void __launch_bounds__(kScanThreads) k_flag_count(long long n, const uint8_t* __restrict__ flag,
                                                             int* __restrict__ bcount) {
    const long long i = (long long)blockIdx.x * kScanThreads + threadIdx.x;
    const int c = __syncthreads_count(i < n && flag[i]);
    if (threadIdx.x == 0) bcount[blockIdx.x] = c;
}

__global__ void __launch_bounds__(kScanThreads) k_flag_compact(long long n, const uint8_t* __restrict__ flag,
                                                               const int* __restrict__ bcount, int* __restrict__ map,
                                                               int* __restrict__ list, int cap, int* __restrict__ count) {
    __shared__ int s_w[kScanThreads / 32];
    __shared__ int s_base;
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    // base: the flagged items of all earlier blocks
    int acc = 0;
    for (int b = t; b < (int)blockIdx.x; b += kScanThreads) acc += bcount[b];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (l == 0) s_w[w] = acc;
    __syncthreads();
    if (t == 0) {
        int sum = 0;
        for (int q = 0; q < kScanThreads / 32; q++) sum += s_w[q];
        s_base = sum;
    }
    __syncthreads();
    const long long i = (long long)blockIdx.x * kScanThreads + t;
    const bool f = i < n && flag[i];
    const unsigned m = __ballot_sync(0xffffffffu, f);
    s_w[w] = __popc(m);  // s_w is free again after the barrier above
    __syncthreads();
    int before = 0;
    for (int q = 0; q < w; q++) before += s_w[q];
    const int r = s_base + before + __popc(m & ((1u << l) - 1u));
    if (i < n) {
        map[i] = f ? r : -1;
        if (f && r < cap) list[r] = (int)i;
    }
    if (blockIdx.x == gridDim.x - 1 && t == kScanThreads - 1) {
        int tot = 0;
        for (int q = 0; q < kScanThreads / 32; q++) tot += s_w[q];
        *count = s_base + tot;
    }
}

static int flag_compact(long long n, const uint8_t* flag, int* bcount, int* map, int* list, int cap, int* count,
                        cudaStream_t st) {
    const unsigned nb = (unsigned)((n + kScanThreads - 1) / kScanThreads);
    pf::count_launch(2);
    k_flag_count<<<nb, kScanThreads, 0, st>>>(n, flag, bcount);
    k_flag_compact<<<nb, kScanThreads, 0, st>>>(n, flag, bcount, map, list, cap, count);
    PF_LAUNCH_CHECK("flag compaction launch");
    return PF_OK;
}

// Ehat of every coarse element, element-major Eh[e * 8 + k] (one 32-byte (FP32) or 64-byte
// (FP64) run per element, read with vector loads)
template <typename T>
__global__ void k_coarse_ehat(int NXc, int NYc, int NZc, const double* __restrict__ E, const int* __restrict__ dmap,
                              T* __restrict__ Eh) {
    const long long ne = (long long)NXc * NYc * NZc;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int ez = (int)(e % NZc), ey = (int)((e / NZc) % NYc), ex = (int)(e / ((long long)NZc * NYc));
    const int NYf = 2 * NYc, NZf = 2 * NZc;
    double c[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int fx = 2 * ex + (q & 1), fy = 2 * ey + ((q >> 1) & 1), fz = 2 * ez + ((q >> 2) & 1);
        c[q] = E[((long long)fx * NYf + fy) * NZf + fz];
    }
    // 8-point Walsh-Hadamard transform over the child bits (x = bit 0)
#pragma unroll
    for (int b = 1; b < 8; b <<= 1)
#pragma unroll
        for (int q = 0; q < 8; q++)
            if (!(q & b)) {
                const double lo = c[q], hi = c[q | b];
                c[q] = lo + hi;
                c[q | b] = lo - hi;
            }
    const int d = dmap ? dmap[e] : -1;
    if (d >= 0) c[0] = -(double)d - 1.0;
#pragma unroll
    for (int q = 0; q < 8; q++) Eh[e * 8 + q] = (T)c[q];
}

template <int DIM>
struct GridC {
    int nel[3], nn[3];
};

__device__ __forceinline__ long long fnode(const GridC<3>& g, int i, int j, int k) {
    return (long long)k + (long long)g.nn[2] * (i + (long long)g.nn[0] * j);
}
__device__ __forceinline__ double hp(int d) { return d == 0 ? 1.0 : d == 1 ? 0.5 : d == 2 ? 0.25 : 0.125; }

// Dirty matrices in the physical basis: thread (d, LI, LJ) writes the 3x3 block of corners
// LI, LJ of dirty element dlist[d]: the dirty part of A^[I, J] if this element is the first
// dirty element containing I and J, else 0.  The dirty part: every dirty element containing
// I and J contributes sum_c E_c (Z Phat_c)^T K0 (Z Phat_c) (children with their fine
// constraints masked, as the reference's level-0 Galerkin, mgm.cu:247-447); the identity
// rows are k_ident_rows'.
__global__ void __launch_bounds__(64) k_dirty_blocks(GridC<3> gf, GridC<3> gc, const double* __restrict__ E,
                                                     const uint8_t* __restrict__ mask,
                                                     const uint8_t* __restrict__ elem_flag,
                                                     const int* __restrict__ dlist, int nd,
                                                     const double* __restrict__ K0, double* __restrict__ M) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nd * 64) return;
    const int d = (int)(t >> 6), LI = (int)((t >> 3) & 7), LJ = (int)(t & 7);
    const int e = dlist[d];
    const int NYc = gc.nel[1], NZc = gc.nel[2];
    const int ez = e % NZc, ey = (e / NZc) % NYc, ex = e / (NZc * NYc);
    const int I[3] = {ex + kCXd(LI), ey + kCYd(LI), ez + kCZd(LI)};
    const int J[3] = {ex + kCXd(LJ), ey + kCYd(LJ), ez + kCZd(LJ)};
    // candidate elements containing I and J: per axis lower corner in [lo_a, hi_a]
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
        const int o = J[a] - I[a];
        if (o == 0) {
            lo[a] = I[a] - 1 < 0 ? 0 : I[a] - 1;
            hi[a] = I[a] > gc.nel[a] - 1 ? gc.nel[a] - 1 : I[a];
        } else {
            lo[a] = hi[a] = o > 0 ? I[a] : J[a];
        }
    }
    // owner: the first dirty candidate in element order
    bool owner = false, found = false;
    for (int cx = lo[0]; cx <= hi[0] && !found; cx++)
        for (int cy = lo[1]; cy <= hi[1] && !found; cy++)
            for (int cz = lo[2]; cz <= hi[2] && !found; cz++) {
                const int ce = (cx * NYc + cy) * NZc + cz;
                if (elem_flag[ce]) {
                    owner = ce == e;
                    found = true;
                }
            }
    double blk[9];
    for (int q = 0; q < 9; q++) blk[q] = 0.0;
    if (owner) {
        for (int cx = lo[0]; cx <= hi[0]; cx++)
            for (int cy = lo[1]; cy <= hi[1]; cy++)
                for (int cz = lo[2]; cz <= hi[2]; cz++) {
                    const int ce = (cx * NYc + cy) * NZc + cz;
                    if (!elem_flag[ce]) continue;
                    // local corners of I and J in element (cx, cy, cz)
                    int li = 0, lj = 0;
                    for (int q = 0; q < 8; q++) {
                        if (cx + kCXd(q) == I[0] && cy + kCYd(q) == I[1] && cz + kCZd(q) == I[2]) li = q;
                        if (cx + kCXd(q) == J[0] && cy + kCYd(q) == J[1] && cz + kCZd(q) == J[2]) lj = q;
                    }
                    for (int c = 0; c < 8; c++) {
                        const int fx = 2 * cx + kCXd(c), fy = 2 * cy + kCYd(c), fz = 2 * cz + kCZd(c);
                        const double we = E[((long long)fx * gf.nel[1] + fy) * gf.nel[2] + fz];
                        for (int l = 0; l < 8; l++) {
                            const int nxl = kCXd(c) + kCXd(l), nyl = kCYd(c) + kCYd(l), nzl = kCZd(c) + kCZd(l);
                            const double pl = (1.0 - 0.5 * abs(nxl - 2 * kCXd(li))) *
                                              (1.0 - 0.5 * abs(nyl - 2 * kCYd(li))) *
                                              (1.0 - 0.5 * abs(nzl - 2 * kCZd(li)));
                            if (pl == 0.0) continue;
                            const uint8_t ml = mask[fnode(gf, 2 * cx + nxl, 2 * cy + nyl, 2 * cz + nzl)];
                            for (int l2 = 0; l2 < 8; l2++) {
                                const int nx2 = kCXd(c) + kCXd(l2), ny2 = kCYd(c) + kCYd(l2), nz2 = kCZd(c) + kCZd(l2);
                                const double p2 = (1.0 - 0.5 * abs(nx2 - 2 * kCXd(lj))) *
                                                  (1.0 - 0.5 * abs(ny2 - 2 * kCYd(lj))) *
                                                  (1.0 - 0.5 * abs(nz2 - 2 * kCZd(lj)));
                                if (p2 == 0.0) continue;
                                const uint8_t m2 = mask[fnode(gf, 2 * cx + nx2, 2 * cy + ny2, 2 * cz + nz2)];
                                const double f = we * pl * p2;
                                for (int a = 0; a < 3; a++) {
                                    if (ml & (1 << a)) continue;
                                    for (int b = 0; b < 3; b++) {
                                        if (m2 & (1 << b)) continue;
                                        blk[a * 3 + b] += f * K0[(l * 3 + a) * 24 + l2 * 3 + b];
                                    }
                                }
                            }
                        }
                    }
                }
    }
    double* Md = M + (long long)d * 576;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Md[(LI * 3 + a) * 24 + LJ * 3 + b] = blk[a * 3 + b];
}

// Identity rows of the level-1 Galerkin operator, Phat^T (I - Z) Phat: thread (q, o) writes,
// for identity node n = nlist[q] and neighbour m = n + o (o = dx + 3 dy + 9 dz + 13), the
// three per-component coefficients S[(a * 27 + o) * icap + q] = sum over the fine nodes f
// within one fine spacing of both 2n and 2m whose DOF a is constrained of
// 0.5^|f - 2n|_0 0.5^|f - 2m|_0 (the interpolation weights; mgm.cu:247-447 adds these rows).
template <typename T>
__global__ void k_ident_rows(GridC<3> gf, GridC<3> gc, const uint8_t* __restrict__ mask, const int* __restrict__ nlist,
                             int nq, int icap, T* __restrict__ S) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nq * 27) return;
    const int q = (int)(t / 27), o = (int)(t % 27);
    const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
    const long long n = nlist[q];
    const int nk = (int)(n % gc.nn[2]), ni = (int)((n / gc.nn[2]) % gc.nn[0]);
    const int nj = (int)(n / ((long long)gc.nn[2] * gc.nn[0]));
    const int mi = ni + dx, mj = nj + dy, mk = nk + dz;
    double acc[3] = {0.0, 0.0, 0.0};
    if (mi >= 0 && mj >= 0 && mk >= 0 && mi < gc.nn[0] && mj < gc.nn[1] && mk < gc.nn[2]) {
        for (int di = -1; di <= 1; di++)
            for (int dj = -1; dj <= 1; dj++)
                for (int dk = -1; dk <= 1; dk++) {
                    const int fi = 2 * ni + di, fj = 2 * nj + dj, fk = 2 * nk + dk;
                    if (fi < 0 || fj < 0 || fk < 0 || fi >= gf.nn[0] || fj >= gf.nn[1] || fk >= gf.nn[2]) continue;
                    const int ei = fi - 2 * mi, ej = fj - 2 * mj, ek = fk - 2 * mk;
                    if (ei < -1 || ei > 1 || ej < -1 || ej > 1 || ek < -1 || ek > 1) continue;
                    const uint8_t m = mask[fnode(gf, fi, fj, fk)];
                    if (!m) continue;
                    const double w = hp((di != 0) + (dj != 0) + (dk != 0)) * hp((ei != 0) + (ej != 0) + (ek != 0));
                    for (int a = 0; a < 3; a++)
                        if (m & (1 << a)) acc[a] += w;
                }
    }
    for (int a = 0; a < 3; a++) S[(long long)(a * 27 + o) * icap + q] = (T)acc[a];
}

// Walsh basis: W = T M T^T / 64, stored Wd[(i * 24 + j) * cap + d] (coalesced across the
// dirty elements of a warp)
template <typename T>
__global__ void __launch_bounds__(576) k_dirty_walsh(const double* __restrict__ M, int cap, T* __restrict__ Wd) {
    __shared__ double s_m[576], s_u[576];
    const int d = blockIdx.x, t = threadIdx.x;
    s_m[t] = M[(long long)d * 576 + t];
    __syncthreads();
    {  // U = M T^T: U[l][j] = sum_n M[l][(n, a_j)] walsh(m_j, n)
        const int l = t / 24, j = t % 24, mj = j / 3, aj = j % 3;
        double s = 0.0;
        for (int n = 0; n < 8; n++) {
            int w = 1;
            const int pos[3] = {kCXd(n), kCYd(n), kCZd(n)};
            for (int a = 0; a < 3; a++)
                if ((mj >> a) & 1) w *= pos[a] ? 1 : -1;
            s += w * s_m[l * 24 + n * 3 + aj];
        }
        s_u[t] = s;
    }
    __syncthreads();
    {  // W[i][j] = sum_n walsh(m_i, n) U[(n, a_i)][j] / 64
        const int i = t / 24, j = t % 24, mi = i / 3, ai = i % 3;
        double s = 0.0;
        for (int n = 0; n < 8; n++) {
            int w = 1;
            const int pos[3] = {kCXd(n), kCYd(n), kCZd(n)};
            for (int a = 0; a < 3; a++)
                if ((mi >> a) & 1) w *= pos[a] ? 1 : -1;
            s += w * s_u[(n * 3 + ai) * 24 + j];
        }
        Wd[(long long)t * cap + d] = (T)(s / 64.0);
    }
}

// ---------------------------------------------------------------------------------------
// matvec: register x-march over coarse elements
// ---------------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ T inv_tw(int n, int nn) {
    return (n == 0 || n == nn - 1) ? T(1.0 / 1.5) : T(0.5);
}

// Element operator in the Walsh basis.  glo / ghi: transformed lower / upper faces; eh: the
// element's Ehat (eh[0] < 0 marks a dirty element, index -eh[0] - 1, if the dirty list
// confirms it for element e).  G receives the lower-face outputs plus the carry of the
// previous element; carry the upper-face outputs.
template <typename T>
__device__ __forceinline__ void coarse_element(const T (&glo)[3][2][2], const T (&ghi)[3][2][2], const T (&eh)[8],
                                               int e, const CoarseCoef<T>& cf, const T* __restrict__ Wd,
                                               const int* __restrict__ dlist, int cap, T (&carry)[3][2][2],
                                               T (&G)[3][2][2]) {
    T v[24];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int ym = 0; ym < 2; ym++)
#pragma unroll
            for (int zm = 0; zm < 2; zm++) {
                v[((0 | (ym << 1) | (zm << 2)) * 3) + a] = ghi[a][ym][zm] + glo[a][ym][zm];
                v[((1 | (ym << 1) | (zm << 2)) * 3) + a] = ghi[a][ym][zm] - glo[a][ym][zm];
            }
    // a negative Ehat_0 is a dirty marker only if the dirty list confirms it (densities that
    // are themselves negative can make Ehat_0 < 0 on a clean element)
    int d = 0;
    bool dirty = false;
    if (eh[0] < T(0) && cap > 0) {
        const T md = -eh[0] - T(1);
        if (md >= T(0) && md < T(cap)) {
            d = (int)md;
            dirty = dlist[d] == e;
        }
    }
    // outputs slot by slot (component a, y-mode, z-mode; x-modes 0 and 1), folded into G.
    // FP32: one branch per element between the explicit and the structured matrix; FP64
    // (254 registers) branches per output, which keeps it free of spills
    if (sizeof(T) == 4 && dirty) {
        const T* wd = Wd + d;
        Unroll<12>::run([&](auto S) {
            constexpr int slot = decltype(S)::value;
            constexpr int a = slot / 4, ym = (slot >> 1) & 1, zm = slot & 1;
            constexpr int i0 = (((ym << 1) | (zm << 2)) * 3) + a, i1 = ((1 | (ym << 1) | (zm << 2)) * 3) + a;
            T z0 = T(0), z1 = T(0);
#pragma unroll
            for (int j = 0; j < 24; j++) z0 = fma(wd[(long long)(i0 * 24 + j) * cap], v[j], z0);
#pragma unroll
            for (int j = 0; j < 24; j++) z1 = fma(wd[(long long)(i1 * 24 + j) * cap], v[j], z1);
            G[a][ym][zm] = (z0 - z1) + carry[a][ym][zm];
            carry[a][ym][zm] = z0 + z1;
        });
        return;
    }
    Unroll<12>::run([&](auto S) {
        constexpr int slot = decltype(S)::value;
        constexpr int a = slot / 4, ym = (slot >> 1) & 1, zm = slot & 1;
        T zx[2];
        Unroll<2>::run([&](auto X) {
            constexpr int xm = decltype(X)::value;
            constexpr int i = ((xm | (ym << 1) | (zm << 2)) * 3) + a;
            T acc = T(0);
            if (sizeof(T) == 8 && dirty) {
                const T* w = Wd + (long long)(i * 24) * cap + d;
#pragma unroll
                for (int j = 0; j < 24; j++) acc = fma(w[(long long)j * cap], v[j], acc);
            } else if constexpr (i >= 3) {
                Unroll<8>::run([&](auto K) {
                    constexpr int k = decltype(K)::value;
                    constexpr int q = wclass(i) ^ k;
                    constexpr int j0 = wslot(q, 0), j1 = wslot(q, 1), j2 = wslot(q, 2);
                    constexpr int c0 = coarse_pat(i, j0), c1 = coarse_pat(i, j1), c2 = coarse_pat(i, j2);
                    if constexpr (c0 >= 0 || c1 >= 0 || c2 >= 0) {
                        T t = T(0);
                        if constexpr (c0 >= 0) t = fma(cf.b[c0 < 0 ? 0 : c0], v[j0], t);
                        if constexpr (c1 >= 0) t = fma(cf.b[c1 < 0 ? 0 : c1], v[j1], t);
                        if constexpr (c2 >= 0) t = fma(cf.b[c2 < 0 ? 0 : c2], v[j2], t);
                        acc = fma(eh[k], t, acc);
                    }
                });
            }
            zx[xm] = acc;
        });
        G[a][ym][zm] = (zx[0] - zx[1]) + carry[a][ym][zm];
        carry[a][ym][zm] = zx[0] + zx[1];
    });
}

// identity rows of owned node (x, y, z), index q: sum over its 27 neighbours m of
// S(a, m) (D u)_m per component a
template <typename T>
__device__ __forceinline__ void coarse_ident(int x, int y, int z, int nx, int ny, int nz, int q, int icap,
                                             const T* __restrict__ S, const T* __restrict__ u, T (&out)[3]) {
    T acc[3] = {T(0), T(0), T(0)};
#pragma unroll 1
    for (int o = 0; o < 27; o++) {
        const int mx = x + o % 3 - 1, my = y + (o / 3) % 3 - 1, mz = z + o / 9 - 1;
        if (mx < 0 || my < 0 || mz < 0 || mx >= nx || my >= ny || mz >= nz) continue;
        const long long m = (long long)mz + (long long)nz * (mx + (long long)nx * my);
        const T dm = inv_tw<T>(mx, nx) * inv_tw<T>(my, ny) * inv_tw<T>(mz, nz);
        for (int a = 0; a < 3; a++) acc[a] = fma(S[(long long)(a * 27 + o) * icap + q], u[3 * m + a] * dm, acc[a]);
    }
    for (int a = 0; a < 3; a++) out[a] = acc[a];
}

// RW element rows per warp: lanes are RW segments of L = 32 / RW along z (shuffles of width L),
// so a z-tile owns L - 2 node columns; RW = 2 wastes fewer lanes when the level's z extent
// is just above a multiple of 30 (level 1 of a 256x128x128 grid: 65 node columns).
template <typename T, int NW, int MINB, int MODE, int RW>
__global__ void __launch_bounds__(NW * 32, MINB)
    k_coarse_matvec(int NX, int NY, int NZ, int CXc, const T* __restrict__ u, const T* __restrict__ Eh,
                    const T* __restrict__ Wd, const int* __restrict__ dlist, int cap, const CoarseCoef<T> cf,
                    Epi<T> epi, const uint8_t* __restrict__ nflag, const int* __restrict__ nmap,
                    const T* __restrict__ S, int icap) {
    pdl_wait();
    pdl_trigger();
    constexpr int L = 32 / RW, NR = NW * RW, TY = NR - 1;  // lanes per row, rows, owned rows
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ T s_q[2][3][NR][L];
    if (epi.skip && *epi.skip) return;
    constexpr bool need_b = MODE != PF_EPI_STORE, need_x = MODE == PF_EPI_JACOBI || MODE == PF_EPI_JACOBI_ADD;
    constexpr bool need_xa = MODE == PF_EPI_JACOBI_ADD;
    const int nx = NX + 1, ny = NY + 1, nz = NZ + 1;
    const int tid = threadIdx.x, w = (tid >> 5) * RW + (tid & 31) / L, l = tid % L;  // w: row, l: lane in row
    const int kz0 = blockIdx.x * (L - 2), jy0 = blockIdx.y * TY, ix0 = blockIdx.z * CXc;
    const int je = jy0 - 1 + w, kc = kz0 - 1 + l;
    const bool col_ok = kc >= 0 && kc < nz;
    const bool ok0 = col_ok && je >= 0 && je < ny, ok1 = col_ok && je + 1 < ny;
    const bool elem_ok = l < L - 1 && je >= 0 && je < NY && kc >= 0 && kc < NZ;
    const bool owner = w < TY && l < L - 2 && je + 1 < ny && kc + 1 < nz;
    const int rows = nz * nx;
    const int n0 = kc + rows * je;
    const int n1 = n0 + rows;
    const int eplane = NY * NZ;
    const int e0 = je * NZ + kc;
    // D = diag(1/tw): per-axis factors of this lane's node column and the two node rows
    const T sz = inv_tw<T>(kc, nz), sy0 = inv_tw<T>(je, ny), sy1 = inv_tw<T>(je + 1, ny);
    const T s0 = sz * sy0, s1 = sz * sy1;
    const T so = inv_tw<T>(kc + 1, nz) * sy1;  // owned node (je + 1, kc + 1), without x
    const T wgt = epi_omega(epi);

    auto load = [&](int p, T (&v)[2][3]) {
        const bool pok = p >= 0 && p < nx;
        const int a0 = n0 + nz * p, a1 = n1 + nz * p;
        const T sx = pok ? inv_tw<T>(p, nx) : T(0);
        if (pok && ok0) {
#pragma unroll
            for (int c = 0; c < 3; c++) v[0][c] = u[3 * a0 + c] * (sx * s0);
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) v[0][c] = T(0);
        }
        if (pok && ok1) {
#pragma unroll
            for (int c = 0; c < 3; c++) v[1][c] = u[3 * a1 + c] * (sx * s1);
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) v[1][c] = T(0);
        }
    };
    auto face = [&](const T (&v)[2][3], T (&g)[3][2][2]) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T s = v[1][c] + v[0][c], dd = v[1][c] - v[0][c];
            const T sn = __shfl_down_sync(FULL, s, 1, L), dn = __shfl_down_sync(FULL, dd, 1, L);
            g[c][0][0] = s + sn;
            g[c][0][1] = sn - s;
            g[c][1][0] = dd + dn;
            g[c][1][1] = dn - dd;
        }
    };
    auto eload = [&](int ie, T (&eh)[8]) {
        const bool ok = elem_ok && ie >= 0 && ie < NX;
        const long long e = (long long)e0 + (long long)eplane * ie;
        if (ok) {
            if constexpr (sizeof(T) == 4) {
                const float4* p = reinterpret_cast<const float4*>(Eh + e * 8);
                const float4 a = p[0], b = p[1];
                eh[0] = a.x, eh[1] = a.y, eh[2] = a.z, eh[3] = a.w;
                eh[4] = b.x, eh[5] = b.y, eh[6] = b.z, eh[7] = b.w;
            } else {
                const double2* p = reinterpret_cast<const double2*>(Eh + e * 8);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const double2 a = p[k];
                    eh[2 * k] = a.x, eh[2 * k + 1] = a.y;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) eh[k] = T(0);
        }
    };

    T carry[3][2][2];
    auto step = [&](int s, T (&gl)[3][2][2], T (&gh)[3][2][2], T (&v)[2][3], T (&eh)[8]) {
        const int ie = ix0 - 1 + s;
        face(v, gh);
        if (s < CXc) load(ie + 2, v);
        const bool out_now = owner && s >= 1 && ie < nx;
        const int no = n1 + 1 + nz * ie;
        T G[3][2][2];
        coarse_element<T>(gl, gh, eh, e0 + eplane * ie, cf, Wd, dlist, cap, carry, G);
        if (s < CXc) eload(ie + 1, eh);
        T pb[3], px[3], pd[3], pa[3];
        if (out_now) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if constexpr (need_b) pb[c] = epi.b[3 * no + c];
                if constexpr (need_x) px[c] = epi.x[3 * no + c];
                if constexpr (need_x) pd[c] = epi.dinv[3 * no + c];
                if constexpr (need_xa) pa[c] = epi.xadd[3 * no + c];
            }
        }
        T P1[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T r0a = G[c][0][0] - G[c][1][0], r0b = G[c][0][1] - G[c][1][1];
            const T r1a = G[c][0][0] + G[c][1][0], r1b = G[c][0][1] + G[c][1][1];
            const T lo0 = r0a - r0b, up0 = r0a + r0b, lo1 = r1a - r1b, up1 = r1a + r1b;
            P1[c] = up1 + __shfl_down_sync(FULL, lo1, 1, L);
            s_q[s & 1][c][w][l] = up0 + __shfl_down_sync(FULL, lo0, 1, L);
        }
        __syncthreads();
        if (out_now) {
            const T sc = so * inv_tw<T>(ie, nx);
            T id[3] = {T(0), T(0), T(0)};
            if (nflag && nflag[no]) coarse_ident<T>(ie, je + 1, kc + 1, nx, ny, nz, nmap[no], icap, S, u, id);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const T y = (P1[c] + s_q[s & 1][c][w + 1][l] + id[c]) * sc;
                T o = y;
                if constexpr (MODE == PF_EPI_RESID) {
                    o = pb[c] - y;
                } else if constexpr (MODE == PF_EPI_JACOBI) {
                    o = px[c] + wgt * pd[c] * (pb[c] - y);
                } else if constexpr (MODE == PF_EPI_JACOBI_ADD) {
                    o = pa[c] + px[c] + wgt * pd[c] * (pb[c] - y);
                }
                epi.out[3 * no + c] = o;
            }
        }
    };

    T gA[3][2][2], gB[3][2][2];
    T vA[2][3];
    T eh[8];
    load(ix0 - 1, vA);
    face(vA, gA);
    load(ix0, vA);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) carry[c][a][b] = T(0);
    eload(ix0 - 1, eh);
    for (int s = 0; s <= CXc; s++) {
        step(s, gA, gB, vA, eh);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 2; b++) gA[c][a][b] = gB[c][a][b];
    }
}

// FP64: 8 warps, 1 block per SM (the operator holds 24 Walsh values and 8 Ehat in
// registers); FP32: 8 warps, 2 blocks per SM (measured: 74.7 us per 256x128x128 level-1
// launch against 81.9 us for one block of 16 warps, whose halo rows are fewer but whose
// step barrier holds all 16 warps)
template <typename T>
struct CoarseShape {  // warps per block (NW - 1 owned element rows) and blocks per SM
    static constexpr int NW = 8;
    static constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
};

// element rows per warp (1 or 2): the one with fewer warp-rows of lanes per x-plane
template <typename T>
static int coarse_rows_per_warp(const Grid& g) {
    if (sizeof(T) != 4) return 1;
    constexpr int NW = CoarseShape<T>::NW;
    long long best = -1;
    int pick = 1;
    for (int rw = 1; rw <= 2; rw++) {
        const int L = 32 / rw, nr = NW * rw;
        const long long cost = (long long)((g.nn[2] + L - 3) / (L - 2)) * ((g.nn[1] + nr - 2) / (nr - 1)) * NW;
        if (best < 0 || cost < best) {
            best = cost;
            pick = rw;
        }
    }
    return pick;
}

template <typename T>
static void coarse_launch_dims(const Grid& g, dim3* grid, int* CXc, int rw) {
    constexpr int NW = CoarseShape<T>::NW;
    const int ny = g.nn[1], nz = g.nn[2], nx = g.nn[0];
    const int L = 32 / rw, nr = NW * rw;
    const int tz = (nz + L - 3) / (L - 2), ty = (ny + nr - 2) / (nr - 1);
    const long long slots = (long long)kNumSM * CoarseShape<T>::MINB;
    const long long cols = (long long)tz * ty;
    int best = 2;
    long long best_cost = -1;
    for (int cx = 2; cx <= 64; cx++) {
        const long long nb = cols * ((nx + cx - 1) / cx);
        const long long cost = ((nb + slots - 1) / slots) * (cx + 1);
        if (best_cost < 0 || cost <= best_cost) {
            best_cost = cost;
            best = cx;
        }
    }
    *CXc = best;
    *grid = dim3(tz, ty, (nx + best - 1) / best);
}

template <typename T, int MODE, int RW>
static int coarse_launch(dim3 grid, int cx, const Grid& g, const T* u, const CoarseOp* c, const CoarseCoef<T>& cf,
                         const Epi<T>& epi, cudaStream_t st) {
    constexpr int NW = CoarseShape<T>::NW, MINB = CoarseShape<T>::MINB;
    const uint8_t* nflag = c->nident > 0 ? c->nflag : nullptr;
    PF_CUDA(launch_pdl(k_coarse_matvec<T, NW, MINB, MODE, RW>, grid, dim3(NW * 32), 0, st, g.nel[0], g.nel[1],
                       g.nel[2], cx, u, (const T*)c->Eh, (const T*)c->Wd, (const int*)c->dlist, c->cap, cf, epi,
                       nflag, (const int*)c->nmap, (const T*)c->S, c->icap));
    return PF_OK;
}

template <typename T>
int launch_coarse_matvec(const CoarseOp* c, const Grid& g, const T* u, const Epi<T>& epi, cudaStream_t st) {
    if (epi.dot_partial) return fail(PF_UNSUPPORTED, "coarse element matvec: no fused dot");
    CoarseCoef<T> cf;
    for (int q = 0; q < kCoarseCoefs; q++) cf.b[q] = (T)c->coef[q];
    const int rw = coarse_rows_per_warp<T>(g);
    dim3 grid;
    int cx;
    coarse_launch_dims<T>(g, &grid, &cx, rw);
    pf::count_launch();
#define PF_COARSE(M)                                                               \
    return rw == 2 ? coarse_launch<T, M, sizeof(T) == 4 ? 2 : 1>(grid, cx, g, u, c, cf, epi, st) \
                   : coarse_launch<T, M, 1>(grid, cx, g, u, c, cf, epi, st)
    switch (epi.mode) {
        case PF_EPI_STORE:
            PF_COARSE(PF_EPI_STORE);
        case PF_EPI_RESID:
            PF_COARSE(PF_EPI_RESID);
        case PF_EPI_JACOBI:
            PF_COARSE(PF_EPI_JACOBI);
        default:
            PF_COARSE(PF_EPI_JACOBI_ADD);
    }
#undef PF_COARSE
}
template int launch_coarse_matvec<double>(const CoarseOp*, const Grid&, const double*, const Epi<double>&,
                                          cudaStream_t);
template int launch_coarse_matvec<float>(const CoarseOp*, const Grid&, const float*, const Epi<float>&,
                                         cudaStream_t);

// ---------------------------------------------------------------------------------------
// object lifetime and setup
// ---------------------------------------------------------------------------------------
static int calloc_dev(void** p, size_t bytes) {
    if (cudaMalloc(p, bytes ? bytes : 8) != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(PF_NO_MEMORY, "device allocation of %zu bytes failed", bytes);
    }
    return PF_OK;
}

int coarse_create(const Op* op, int fp32, CoarseOp** out) {
    *out = nullptr;
    CoarseOp* c = new CoarseOp();
    int s = coarse_factorise(op, c->coef);
    if (s) {
        cudaGetLastError();
        delete c;
        return s;
    }
    c->fine = op->grid;
    c->g = coarse_grid(op->grid);
    c->tsize = fp32 ? 4 : 8;
    const long long ne = c->g.n_elem;
    s = calloc_dev(&c->Eh, (size_t)ne * 8 * c->tsize);
    s = s ? s : calloc_dev((void**)&c->dmap, (size_t)ne * sizeof(int));
    s = s ? s : calloc_dev((void**)&c->nmap, (size_t)c->g.n_nodes * sizeof(int));
    s = s ? s : calloc_dev((void**)&c->count, 2 * sizeof(int));
    {
        const long long nmax = ne > c->g.n_nodes ? ne : c->g.n_nodes;
        s = s ? s : calloc_dev((void**)&c->bcount, (size_t)((nmax + kScanThreads - 1) / kScanThreads) * sizeof(int));
    }
    if (!s && cudaMallocHost((void**)&c->h_count, 2 * sizeof(int)) != cudaSuccess) s = fail(PF_NO_MEMORY, "pinned alloc");
    if (s) {
        coarse_destroy(c);
        return s;
    }
    *out = c;
    return PF_OK;
}

void coarse_destroy(CoarseOp* c) {
    if (!c) return;
    for (void* p : {c->Eh, (void*)c->dmap, (void*)c->dlist, (void*)c->M, c->Wd, (void*)c->count, (void*)c->nmap,
                    (void*)c->nlist, c->S, (void*)c->bcount})
        if (p) cudaFree(p);
    if (c->h_count) cudaFreeHost(c->h_count);
    delete c;
}

static GridC<3> gridc(const Grid& g) {
    GridC<3> r;
    for (int a = 0; a < 3; a++) {
        r.nel[a] = g.nel[a];
        r.nn[a] = g.nn[a];
    }
    return r;
}

// Ehat and the dirty matrices for densities E (FP64) and the fine node mask.  The dirty
// list is recounted on every call; the host waits for the count (one int) and grows the
// dirty storage when it no longer fits.
int coarse_setup(CoarseOp* c, const double* E, const uint8_t* mask, const uint8_t* elem_flag,
                 const uint8_t* node_flag, const double* K0_dev, cudaStream_t st, bool* realloc) {
    *realloc = false;
    const Grid& gc = c->g;
    const long long ne = gc.n_elem;
    if (ne >= (1LL << 31) || gc.n_nodes >= (1LL << 31)) return fail(PF_BAD_ARG, "coarse grid too large");
    int nd = 0, ni = 0;
    c->nflag = node_flag;
    if (mask) {
        for (int pass = 0; pass < 2; pass++) {
            int s = flag_compact(ne, elem_flag, c->bcount, c->dmap, c->dlist, c->cap, c->count, st);
            s = s ? s : flag_compact(gc.n_nodes, node_flag, c->bcount, c->nmap, c->nlist, c->icap, c->count + 1, st);
            if (s) return s;
            PF_CUDA(cudaMemcpyAsync(c->h_count, c->count, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
            PF_CUDA(cudaStreamSynchronize(st));
            nd = c->h_count[0];
            ni = c->h_count[1];
            if (nd <= c->cap && ni <= c->icap) break;
            if (nd >= (1 << 24)) return fail(PF_UNSUPPORTED, "coarse operator: %d dirty elements (limit 2^24)", nd);
            if (nd > c->cap) {
                for (void* p : {(void*)c->dlist, (void*)c->M, c->Wd})
                    if (p) cudaFree(p);
                c->dlist = nullptr;
                c->M = nullptr;
                c->Wd = nullptr;
                const int cap = nd + nd / 4 + 32;
                int s = calloc_dev((void**)&c->dlist, (size_t)cap * sizeof(int));
                s = s ? s : calloc_dev((void**)&c->M, (size_t)cap * 576 * sizeof(double));
                s = s ? s : calloc_dev(&c->Wd, (size_t)cap * 576 * c->tsize);
                if (s) {
                    c->cap = 0;
                    return s;
                }
                c->cap = cap;
            }
            if (ni > c->icap) {
                for (void* p : {(void*)c->nlist, c->S})
                    if (p) cudaFree(p);
                c->nlist = nullptr;
                c->S = nullptr;
                const int icap = ni + ni / 4 + 32;
                int s = calloc_dev((void**)&c->nlist, (size_t)icap * sizeof(int));
                s = s ? s : calloc_dev(&c->S, (size_t)icap * 81 * c->tsize);
                if (s) {
                    c->icap = 0;
                    return s;
                }
                c->icap = icap;
            }
            *realloc = true;
        }
    }
    c->nident = ni;
    c->ndirty = nd;
    const unsigned nb = (unsigned)((ne + 255) / 256);
    pf::count_launch();
    if (c->tsize == 4)
        k_coarse_ehat<float><<<nb, 256, 0, st>>>(gc.nel[0], gc.nel[1], gc.nel[2], E, mask ? c->dmap : nullptr,
                                                 (float*)c->Eh);
    else
        k_coarse_ehat<double><<<nb, 256, 0, st>>>(gc.nel[0], gc.nel[1], gc.nel[2], E, mask ? c->dmap : nullptr,
                                                  (double*)c->Eh);
    PF_LAUNCH_CHECK("coarse ehat launch");
    if (nd > 0) {
        pf::count_launch(2);
        k_dirty_blocks<<<(unsigned)(((long long)nd * 64 + 63) / 64), 64, 0, st>>>(
            gridc(c->fine), gridc(gc), E, mask, elem_flag, c->dlist, nd, K0_dev, c->M);
        PF_LAUNCH_CHECK("dirty blocks launch");
        if (c->tsize == 4)
            k_dirty_walsh<float><<<nd, 576, 0, st>>>(c->M, c->cap, (float*)c->Wd);
        else
            k_dirty_walsh<double><<<nd, 576, 0, st>>>(c->M, c->cap, (double*)c->Wd);
        PF_LAUNCH_CHECK("dirty walsh launch");
    }
    if (ni > 0) {
        pf::count_launch();
        const unsigned nbi = (unsigned)(((long long)ni * 27 + 255) / 256);
        if (c->tsize == 4)
            k_ident_rows<float><<<nbi, 256, 0, st>>>(gridc(c->fine), gridc(gc), mask, c->nlist, ni, c->icap,
                                                     (float*)c->S);
        else
            k_ident_rows<double><<<nbi, 256, 0, st>>>(gridc(c->fine), gridc(gc), mask, c->nlist, ni, c->icap,
                                                      (double*)c->S);
        PF_LAUNCH_CHECK("identity rows launch");
    }
    return PF_OK;
}

}  // namespace pf
