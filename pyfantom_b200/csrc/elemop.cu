// Element operator of the structured SIMP stiffness K(E) = sum_e E_e K0_e:
// matvec (with Dirichlet identity rows), diagonal and -u_e^T K0 u_e.
//
// H8 factorisation.  Both axis-aligned reflections of a box element map the element onto
// itself, so K0 commutes with them.  In the Walsh basis of the 2x2x2 corners
// (v = T u with T[(m,c),(l,c')] = delta_cc' prod_axis (m_axis ? +-1 : 1)) K0 becomes
// block diagonal: B = T K0 T^T / 64 has eight 3x3 blocks, one per parity class
// p = (px,py,pz), coupling component c in mode p ^ e_c.  K0 u = T^T B T u costs
// 3 butterfly stages forward, 8 3x3 blocks and 3 stages back (~150 flops for a cube
// element, against 576 multiply-adds for the dense 24x24 product).  The matvec kernel
// marches along x: warps cover element rows in y, lanes cover element columns in z (the
// contiguous node axis); each lane reads its node column of two rows straight into
// registers, the y/z stages of a face are done once and shared by the two elements on
// either side of it along x, z neighbours are exchanged by shuffles and rows through one
// shared-memory exchange per step.  Owner-computes: each node is written once, no atomics,
// fixed summation order.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "elemop.cuh"

namespace pf {

// ---------------------------------------------------------------------------------------
// host: transform-block factorisation of K0
// ---------------------------------------------------------------------------------------
static const int kCX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int kCY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int kCZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

// The 33 distinct nonzeros of the eight symmetric 3x3 class blocks of an isotropic box
// element: class p, row i, column j (upper triangle of each block's nonzero pattern).
static const int kCoefP[33] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 3, 4,
                               4, 4, 5, 5, 5, 5, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7};
static const int kCoefI[33] = {0, 0, 0, 1, 1, 2, 1, 1, 2, 0, 0, 2, 0, 0, 1, 2, 0,
                               0, 1, 0, 0, 2, 1, 1, 1, 2, 0, 0, 0, 0, 1, 1, 2};
static const int kCoefJ[33] = {0, 1, 2, 1, 2, 2, 1, 2, 2, 0, 2, 2, 0, 1, 1, 2, 0,
                               1, 1, 0, 2, 2, 1, 1, 2, 2, 0, 0, 1, 2, 1, 2, 2};

static bool h8_coef_nonzero(int p, int i, int j) {
    for (int q = 0; q < 33; q++)
        if (kCoefP[q] == p && ((kCoefI[q] == i && kCoefJ[q] == j) || (kCoefI[q] == j && kCoefJ[q] == i))) return true;
    return false;
}

static int walsh(int m, int l, int dim) {
    int pos[3] = {kCX[l], kCY[l], dim == 3 ? kCZ[l] : 0};
    int s = 1;
    for (int a = 0; a < dim; a++)
        if ((m >> a) & 1) s *= pos[a] ? 1 : -1;
    return s;
}

int op_factorise(Op* op) {
    const int dim = op->grid.dim, nc = dim == 3 ? 8 : 4, nd = nc * dim;
    // T (nd x nd): row (m, c), column (l, c')
    std::vector<double> T(nd * nd, 0.0), tmp(nd * nd, 0.0), B(nd * nd, 0.0);
    for (int m = 0; m < nc; m++)
        for (int l = 0; l < nc; l++)
            for (int c = 0; c < dim; c++) T[(m * dim + c) * nd + l * dim + c] = walsh(m, l, dim);
    // B = T K0 T^T / nc^2
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++) {
            double s = 0;
            for (int k = 0; k < nd; k++) s += T[i * nd + k] * op->K0[k * nd + j];
            tmp[i * nd + j] = s;
        }
    double bmax = 0.0;
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++) {
            double s = 0;
            for (int k = 0; k < nd; k++) s += tmp[i * nd + k] * T[j * nd + k];
            B[i * nd + j] = s / double(nc * nc);
            bmax = fmax(bmax, fabs(B[i * nd + j]));
        }
    // extract class blocks and verify that nothing lies outside them
    std::vector<char> used(nd * nd, 0);
    for (int p = 0; p < nc; p++)
        for (int c = 0; c < dim; c++)
            for (int c2 = 0; c2 < dim; c2++) {
                int row = (p ^ (1 << c)) * dim + c, col = (p ^ (1 << c2)) * dim + c2;
                op->blk[p][c][c2] = B[row * nd + col];
                used[row * nd + col] = 1;
            }
    double off = 0.0;
    for (int i = 0; i < nd * nd; i++)
        if (!used[i]) off = fmax(off, fabs(B[i]));
    if (!(off <= 1e-12 * bmax))
        return fail(PF_UNSUPPORTED,
                    "K0 is not invariant under the element's axis reflections (off-block %.3e vs %.3e)", off, bmax);
    op->sparse = 0;
    op->cube = 0;
    if (dim == 3) {
        // Isotropic box elements: each class block is symmetric and zero outside the
        // pattern below (the rows of the rigid translations vanish, and reflection
        // symmetry decouples the rest), leaving 33 distinct coefficients.
        const double tol = 1e-12 * bmax;
        bool ok = true;
        for (int p = 0; p < 8; p++)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) {
                    if (fabs(op->blk[p][i][j] - op->blk[p][j][i]) > tol) ok = false;
                    if (!h8_coef_nonzero(p, i, j) && fabs(op->blk[p][i][j]) > tol) ok = false;
                }
        if (ok) {
            for (int q = 0; q < 33; q++) op->coef[q] = op->blk[kCoefP[q]][kCoefI[q]][kCoefJ[q]];
            op->sparse = 1;
            // cube element: seven values in the pattern of cube_index()
            const int rep[7] = {0, 1, 7, 12, 15, 27, 28};
            for (int v = 0; v < 7; v++) op->cube_v[v] = op->coef[rep[v]];
            bool cube = true;
            for (int q = 0; q < 33; q++)
                if (fabs(op->coef[q] - op->cube_v[cube_index(q)]) > tol) cube = false;
            op->cube = cube ? 1 : 0;
        }
    }
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// 3D matvec operands
// ---------------------------------------------------------------------------------------
template <typename T>
struct H8Blk {
    T b[8][3][3];
};
template <typename T>
struct H8Coef {
    T c[33];  // the 33 sparse coefficients (CM 1) or the 7 cube values (CM 2)
};

// ---------------------------------------------------------------------------------------
// 3D matvec: register x-march
// ---------------------------------------------------------------------------------------
// One element per thread and step.  Warp w of a block computes element row
// je = jy0 - 1 + w, lane l element column ke = kz0 - 1 + l (lanes 0..30; lane 31 only
// supplies its node column to lane 30).  Each lane reads its own node column of rows je
// and je + 1 straight from global memory into registers one plane ahead (a warp reads 32
// consecutive nodes of a row: coalesced), forms the y stage of the face transform of that
// column and takes the z neighbour's by shuffle, so the forward path uses neither shared
// memory nor a barrier.  On the way back the z neighbour's corner arrives by shuffle and the
// contribution to node row je goes to the warp below through one shared-memory exchange,
// the only barrier of the step.  Warps 0..NW-2 own node rows jy0 .. jy0+NW-2 and lanes
// 0..29 node columns kz0 .. kz0+29.  For a cube element (CM 2) the element's scale is
// folded into the seven coefficient values instead of the 24 transformed inputs.
// Loaded values are never copied between registers before use (a copy would wait for the
// load): the constraint bytes stay separate until the next step and each element scale is
// loaded straight into its register once the current one is spent.  (Unrolling the march by
// two to alternate register sets, or prefetching two planes ahead, measured slower: more
// registers, fewer resident warps.)
// Remainder z-tile: when the last z-tile holds at most 14 node columns (129 = 4 x 30 + 9
// columns at 256x128x128, 97 = 3 x 30 + 7 at 192x96x96) its blocks split every warp into two
// 16-lane segments, each computing its own element row (shuffles of width 16, 14 owned
// columns per segment), so that tile costs half the warp-steps of a full-width one.  Blocks
// 0 .. tzA * tyA - 1 are full-width tiles (z-tile b % tzA, y-tile b / tzA); the blocks after
// them are the half-width y-tiles of the z-tile starting at column tzA * 30.
constexpr int kZTileR = 30;
struct H8Tiles {
    int tzA, tyA;  // full-width z-tiles and y-tiles
    int ncols;     // tile columns: tzA * tyA full-width, then the half-width ones
};

// element scale in the operator precision (E stored in FP64, FP32 or BF16)
template <typename T, typename TE>
__device__ __forceinline__ T elem_scale(TE e) {
    if constexpr (std::is_same<TE, __nv_bfloat16>::value)
        return (T)__bfloat162float(e);
    else
        return (T)e;
}

// Two FP32 values in one 64-bit register pair, operated on by the packed FP32 instructions
// of sm_100 (add/sub/mul/fma .f32x2): the paired fine matvec below runs the element
// operator on two z-neighbouring elements at once (x = the lower element, y = the upper).
// (Its own namespace, so that its fma is found by argument-dependent lookup and does not
// hide the scalar fma of the other kernels in this namespace.)
namespace pk {
struct F2 {
    unsigned long long v;
    __device__ __forceinline__ F2() {}
    __device__ __forceinline__ explicit F2(float s) { asm("mov.b64 %0, {%1, %1};" : "=l"(v) : "f"(s)); }
    __device__ __forceinline__ F2(float a, float b) { asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(a), "f"(b)); }
    __device__ __forceinline__ float x() const {
        float a, b;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
        return a;
    }
    __device__ __forceinline__ float y() const {
        float a, b;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
        return b;
    }
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) {
    F2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    F2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) {
    F2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) {
    F2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
}  // namespace pk
using pk::F2;

// Element operator in the Walsh basis.  glo / ghi: transformed lower / upper faces (yz
// stages done); e: the element's scale.  Returns in G the lower-face outputs plus the
// upper-face outputs of the previous element (carry), and leaves this element's upper-face
// outputs in carry.  Classes are taken in (y, z) parity pairs: the pair p = (0,py,pz),
// (1,py,pz) reads and writes exactly the modes (c=0: py,pz), (c=1: py^1,pz), (c=2: py,pz^1).
template <typename T, int CM>
__device__ __forceinline__ void h8_element(const T (&glo)[3][2][2], const T (&ghi)[3][2][2], T e,
                                           const H8Coef<T>& cf, const volatile T* vb, T (&carry)[3][2][2],
                                           T (&G)[3][2][2]) {
    // x stage of slot (component c, y-mode ym, z-mode zm): A = x-mode 0, B = x-mode 1
#define XST(c, ym, zm, A, B)                                                                  \
    const T A = (CM == 2) ? ghi[c][ym][zm] + glo[c][ym][zm] : e * (ghi[c][ym][zm] + glo[c][ym][zm]); \
    const T B = (CM == 2) ? ghi[c][ym][zm] - glo[c][ym][zm] : e * (ghi[c][ym][zm] - glo[c][ym][zm]);
    // inverse x stage for pair (py, pz): class p0 outputs o0*, class p1 outputs o1*
#define XINV(py, pz, o00, o01, o02, o10, o11, o12)                 \
    G[0][py][pz] = ((o10) - (o00)) + carry[0][py][pz];             \
    carry[0][py][pz] = (o10) + (o00);                              \
    G[1][(py) ^ 1][pz] = ((o01) - (o11)) + carry[1][(py) ^ 1][pz]; \
    carry[1][(py) ^ 1][pz] = (o01) + (o11);                        \
    G[2][py][(pz) ^ 1] = ((o02) - (o12)) + carry[2][py][(pz) ^ 1]; \
    carry[2][py][(pz) ^ 1] = (o02) + (o12);
    if constexpr (CM == 2) {
        // cube element: values a-b, b, c, d, e, f-g, g, each times the element scale
        const T kA = e * cf.c[0], kB = e * cf.c[1], kC = e * cf.c[2], kD = e * cf.c[3];
        const T kE = e * cf.c[4], kF = e * cf.c[5], kG = e * cf.c[6];
        {  // pair (0,0): class 0 circulant on (b0, a1, a2); class 1 [[b,c],[c,b]] on (b1, b2)
            XST(0, 0, 0, a0, b0)
            XST(1, 1, 0, a1, b1)
            XST(2, 0, 1, a2, b2)
            (void)a0;
            const T bs = kB * (b0 + a1 + a2);
            const T o00 = fma(kA, b0, bs), o01 = fma(kA, a1, bs), o02 = fma(kA, a2, bs);
            const T o11 = fma(kB, b1, kC * b2), o12 = fma(kC, b1, kB * b2);
            XINV(0, 0, o00, o01, o02, T(0), o11, o12)
        }
        {  // pair (1,0): class 2 [[b,c],[c,b]] on (b0, a2); class 3 d on (a0, b1), e on b2
            XST(0, 1, 0, a0, b0)
            XST(1, 0, 0, a1, b1)
            XST(2, 1, 1, a2, b2)
            (void)a1;
            const T o00 = fma(kB, b0, kC * a2), o02 = fma(kC, b0, kB * a2);
            const T o10 = kD * (a0 + b1);
            const T o12 = kE * b2;
            XINV(1, 0, o00, T(0), o02, o10, o10, o12)
        }
        {  // pair (0,1): class 4 [[b,c],[c,b]] on (b0, a1); class 5 d on (a0, b2), e on b1
            XST(0, 0, 1, a0, b0)
            XST(1, 1, 1, a1, b1)
            XST(2, 0, 0, a2, b2)
            (void)a2;
            const T o00 = fma(kB, b0, kC * a1), o01 = fma(kC, b0, kB * a1);
            const T o10 = kD * (a0 + b2);
            const T o11 = kE * b1;
            XINV(0, 1, o00, o01, T(0), o10, o11, o10)
        }
        {  // pair (1,1): class 6 e on b0, d on (a1, a2); class 7 circulant on (a0, b1, b2)
            XST(0, 1, 1, a0, b0)
            XST(1, 0, 1, a1, b1)
            XST(2, 1, 0, a2, b2)
            const T o00 = kE * b0;
            const T o01 = kD * (a1 + a2);
            const T gs = kG * (a0 + b1 + b2);
            const T o10 = fma(kF, a0, gs), o11 = fma(kF, b1, gs), o12 = fma(kF, b2, gs);
            XINV(1, 1, o00, o01, o01, o10, o11, o12)
        }
    } else if constexpr (CM == 1) {
#define KC(q) cf.c[q]
        {
            XST(0, 0, 0, a0, b0)
            XST(1, 1, 0, a1, b1)
            XST(2, 0, 1, a2, b2)
            (void)a0;
            const T o00 = fma(KC(0), b0, fma(KC(1), a1, KC(2) * a2));
            const T o01 = fma(KC(1), b0, fma(KC(3), a1, KC(4) * a2));
            const T o02 = fma(KC(2), b0, fma(KC(4), a1, KC(5) * a2));
            const T o11 = fma(KC(6), b1, KC(7) * b2);
            const T o12 = fma(KC(7), b1, KC(8) * b2);
            XINV(0, 0, o00, o01, o02, T(0), o11, o12)
        }
        {
            XST(0, 1, 0, a0, b0)
            XST(1, 0, 0, a1, b1)
            XST(2, 1, 1, a2, b2)
            (void)a1;
            const T o00 = fma(KC(9), b0, KC(10) * a2);
            const T o02 = fma(KC(10), b0, KC(11) * a2);
            const T o10 = fma(KC(12), a0, KC(13) * b1);
            const T o11 = fma(KC(13), a0, KC(14) * b1);
            const T o12 = KC(15) * b2;
            XINV(1, 0, o00, T(0), o02, o10, o11, o12)
        }
        {
            XST(0, 0, 1, a0, b0)
            XST(1, 1, 1, a1, b1)
            XST(2, 0, 0, a2, b2)
            (void)a2;
            const T o00 = fma(KC(16), b0, KC(17) * a1);
            const T o01 = fma(KC(17), b0, KC(18) * a1);
            const T o10 = fma(KC(19), a0, KC(20) * b2);
            const T o12 = fma(KC(20), a0, KC(21) * b2);
            const T o11 = KC(22) * b1;
            XINV(0, 1, o00, o01, T(0), o10, o11, o12)
        }
        {
            XST(0, 1, 1, a0, b0)
            XST(1, 0, 1, a1, b1)
            XST(2, 1, 0, a2, b2)
            const T o00 = KC(26) * b0;
            const T o01 = fma(KC(23), a1, KC(24) * a2);
            const T o02 = fma(KC(24), a1, KC(25) * a2);
            const T o10 = fma(KC(27), a0, fma(KC(28), b1, KC(29) * b2));
            const T o11 = fma(KC(28), a0, fma(KC(30), b1, KC(31) * b2));
            const T o12 = fma(KC(29), a0, fma(KC(31), b1, KC(32) * b2));
            XINV(1, 1, o00, o01, o02, o10, o11, o12)
        }
#undef KC
    } else {
        // any reflection-symmetric K0: dense 3x3 class blocks re-read from shared memory
#define BK(p, i, j) vb[(p) * 9 + (i) * 3 + (j)]
#pragma unroll
        for (int pyz = 0; pyz < 4; pyz++) {
            const int py = pyz & 1, pz = pyz >> 1;
            const int p0 = 2 * py + 4 * pz, p1 = p0 + 1;
            const T h0 = e * ghi[0][py][pz], h1 = e * ghi[1][py ^ 1][pz], h2 = e * ghi[2][py][pz ^ 1];
            const T a0 = fma(e, glo[0][py][pz], h0), b0 = fma(-e, glo[0][py][pz], h0);
            const T a1 = fma(e, glo[1][py ^ 1][pz], h1), b1 = fma(-e, glo[1][py ^ 1][pz], h1);
            const T a2 = fma(e, glo[2][py][pz ^ 1], h2), b2 = fma(-e, glo[2][py][pz ^ 1], h2);
            const T o00 = fma(BK(p0, 0, 0), b0, fma(BK(p0, 0, 1), a1, BK(p0, 0, 2) * a2));
            const T o01 = fma(BK(p0, 1, 0), b0, fma(BK(p0, 1, 1), a1, BK(p0, 1, 2) * a2));
            const T o02 = fma(BK(p0, 2, 0), b0, fma(BK(p0, 2, 1), a1, BK(p0, 2, 2) * a2));
            const T o10 = fma(BK(p1, 0, 0), a0, fma(BK(p1, 0, 1), b1, BK(p1, 0, 2) * b2));
            const T o11 = fma(BK(p1, 1, 0), a0, fma(BK(p1, 1, 1), b1, BK(p1, 1, 2) * b2));
            const T o12 = fma(BK(p1, 2, 0), a0, fma(BK(p1, 2, 1), b1, BK(p1, 2, 2) * b2));
            G[0][py][pz] = (o10 - o00) + carry[0][py][pz];
            carry[0][py][pz] = o10 + o00;
            G[1][py ^ 1][pz] = (o01 - o11) + carry[1][py ^ 1][pz];
            carry[1][py ^ 1][pz] = o01 + o11;
            G[2][py][pz ^ 1] = (o02 - o12) + carry[2][py][pz ^ 1];
            carry[2][py][pz ^ 1] = o02 + o12;
        }
#undef BK
    }
#undef XINV
#undef XST
}

template <typename T, typename TE, int NW, int MINB, int CM, int MODE, bool DOT>
__global__ void __launch_bounds__(NW * 32, MINB)
    k_matvec_h8r(int NX, int NY, int NZ, H8Tiles tl, const T* __restrict__ u, const TE* __restrict__ E,
                 const uint8_t* __restrict__ mask, const H8Blk<T> blk, const H8Coef<T> cf, Epi<T> epi) {
    pdl_wait();
    pdl_trigger();
    constexpr int NT = NW * 32;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ T s_q[2][3][NW * 32];  // [w * L + l]
    __shared__ double s_red[NW];
    __shared__ T s_blk[72];
    if (epi.skip && *epi.skip) return;
    constexpr int mode = MODE;
    constexpr bool need_b = mode != PF_EPI_STORE, need_x = mode == PF_EPI_JACOBI || mode == PF_EPI_JACOBI_ADD;
    constexpr bool need_xa = mode == PF_EPI_JACOBI_ADD;
    const int nx = NX + 1, ny = NY + 1, nz = NZ + 1;
    const int tid = threadIdx.x;
    double dot = 0.0;
    if (CM == 0 && tid < 72) s_blk[tid] = blk.b[tid / 9][(tid / 3) % 3][tid % 3];
    if (CM == 0) __syncthreads();
    const volatile T* vb = s_blk;
    // this block's share of the (tile column, node plane) work, node planes contiguous within
    // a column: one march per column segment
    const long long total = (long long)tl.ncols * nx;
    long long wpos = total * blockIdx.x / gridDim.x;
    const long long wend = total * (blockIdx.x + 1) / gridDim.x;
    for (int seg = 0; wpos < wend; seg++) {
    const int col = (int)(wpos / nx), ix0 = (int)(wpos % nx);
    const int CXc = (int)min(wend - wpos, (long long)(nx - ix0));  // node planes ix0 .. ix0 + CXc - 1
    wpos += CXc;
    if (seg > 0) __syncthreads();  // the previous segment's last row exchange is read
    // block-uniform tile shape: L lanes per element row (32, or 16 in the remainder z-tile)
    const int bA = tl.tzA * tl.tyA;
    const bool half = col >= bA;
    const int L = half ? 16 : 32, TY = (half ? 2 * NW : NW) - 1;
    const int w = half ? tid >> 4 : tid >> 5, l = tid & (L - 1);
    const int zt = half ? tl.tzA : col % max(tl.tzA, 1);
    const int yt = half ? col - bA : col / max(tl.tzA, 1);
    const int kz0 = zt * kZTileR, jy0 = yt * TY;
    const int je = jy0 - 1 + w, kc = kz0 - 1 + l;  // element row; node column of its lower z corner
    const bool col_ok = kc >= 0 && kc < nz;
    const bool ok0 = col_ok && je >= 0 && je < ny, ok1 = col_ok && je + 1 < ny;
    const bool elem_ok = l < L - 1 && je >= 0 && je < NY && kc >= 0 && kc < NZ;
    const bool owner = w < TY && l < L - 2 && je + 1 < ny && kc + 1 < nz;
    // 32-bit node and element indices (grid validation keeps 3 * nodes below 2^31)
    const int rows = nz * nx;        // nodes per node row (y)
    const int n0 = kc + rows * je;   // node (je, 0, kc): rows je, je + 1 advance by nz per plane
    const int n1 = n0 + rows;
    const int eplane = NY * NZ;      // elements per element plane (x)
    const int e0 = je * NZ + kc;     // element (0, je, kc)
    const bool has_mask = mask != nullptr;
    const T wgt = epi_omega(epi);

    // node values of this lane's column in rows je, je+1 of plane p (zero outside the mesh)
    // and the two constraint bytes; nothing here waits for the loads
    auto load = [&](int p, T (&v)[2][3], int& m0, int& m1) {
        const bool pok = p >= 0 && p < nx;
        const int a0 = n0 + nz * p, a1 = n1 + nz * p;
        m0 = 0;
        m1 = 0;
        if (pok && ok0) {
#pragma unroll
            for (int c = 0; c < 3; c++) v[0][c] = u[3 * a0 + c];
            if (has_mask) m0 = mask[a0];
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) v[0][c] = T(0);
        }
        if (pok && ok1) {
#pragma unroll
            for (int c = 0; c < 3; c++) v[1][c] = u[3 * a1 + c];
            if (has_mask) m1 = mask[a1];
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++) v[1][c] = T(0);
        }
    };
    // y stage of this column, z stage with the next column's (shuffle): transformed face
    auto face = [&](T (&v)[2][3], int m0, int m1, T (&g)[3][2][2]) {
        if (__any_sync(FULL, m0 | m1)) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if ((m0 >> c) & 1) v[0][c] = T(0);
                if ((m1 >> c) & 1) v[1][c] = T(0);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T s = v[1][c] + v[0][c], d = v[1][c] - v[0][c];
            const T sn = __shfl_down_sync(FULL, s, 1, L), dn = __shfl_down_sync(FULL, d, 1, L);
            g[c][0][0] = s + sn;
            g[c][0][1] = sn - s;
            g[c][1][0] = d + dn;
            g[c][1][1] = dn - d;
        }
    };
    auto escale = [&](int ie) -> T { return (elem_ok && ie >= 0 && ie < NX) ? elem_scale<T>(E[e0 + eplane * ie]) : T(0); };

    // One step (element ie = ix0 - 1 + s).
    //   v, m0, m1: plane ie+1 (loaded one step earlier); refilled with plane ie+2
    //   e: scale of element ie; refilled with that of element ie+1 after its last use
    T carry[3][2][2];
    auto step = [&](int s, T (&gl)[3][2][2], T (&gh)[3][2][2], T (&v)[2][3], int& m0, int& m1, T& e) {
        const int ie = ix0 - 1 + s;
        face(v, m0, m1, gh);
        if (s < CXc) load(ie + 2, v, m0, m1);
        // epilogue operands of the owned node (je+1, ie, kc+1), consumed after the barrier:
        // loaded before the element operator, except the three Jacobi vectors in FP64, which
        // are loaded after it (held across it they would spill)
        const bool out_now = owner && s >= 1 && ie < nx;
        const int no = n1 + 1 + nz * ie;
        T pb[3], px[3], pd[3], pa[3], pt[3];
        int mo = 0;
        constexpr bool late = sizeof(T) == 8 && need_x;
        auto fetch = [&]() {
            if (out_now) {
                if (has_mask) mo = mask[no];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    if constexpr (need_b) pb[c] = epi.b[3 * no + c];
                    if constexpr (need_x) px[c] = epi.x[3 * no + c];
                    if constexpr (need_x) pd[c] = epi.dinv[3 * no + c];
                    if constexpr (need_xa) pa[c] = epi.xadd[3 * no + c];
                    if constexpr (DOT) pt[c] = epi.dot_a[3 * no + c];
                }
            }
        };
        if constexpr (!late) fetch();
        T G[3][2][2];
        h8_element<T, CM>(gl, gh, e, cf, vb, carry, G);
        if constexpr (late) fetch();
        e = (s < CXc) ? escale(ie + 1) : T(0);
        // inverse y and z stages; node (je+1, kc+1) from this lane and the next, the row je
        // part to the warp below
        T P1[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const T r0a = G[c][0][0] - G[c][1][0], r0b = G[c][0][1] - G[c][1][1];
            const T r1a = G[c][0][0] + G[c][1][0], r1b = G[c][0][1] + G[c][1][1];
            const T lo0 = r0a - r0b, up0 = r0a + r0b, lo1 = r1a - r1b, up1 = r1a + r1b;
            P1[c] = up1 + __shfl_down_sync(FULL, lo1, 1, L);
            s_q[s & 1][c][w * L + l] = up0 + __shfl_down_sync(FULL, lo0, 1, L);
        }
        __syncthreads();
        if (out_now) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                T y = P1[c] + s_q[s & 1][c][(w + 1) * L + l];
                if ((mo >> c) & 1) y = u[3 * no + c];
                T o = y;
                if constexpr (mode == PF_EPI_RESID) {
                    o = pb[c] - y;
                } else if constexpr (mode == PF_EPI_JACOBI) {
                    o = px[c] + wgt * pd[c] * (pb[c] - y);
                } else if constexpr (mode == PF_EPI_JACOBI_ADD) {
                    o = pa[c] + px[c] + wgt * pd[c] * (pb[c] - y);
                }
                epi.out[3 * no + c] = o;
                if constexpr (DOT) dot += (double)pt[c] * (double)(epi.dot_of_y ? y : o);
            }
        }
    };

    T gA[3][2][2], gB[3][2][2];
    T vA[2][3];
    int mA0, mA1;
    load(ix0 - 1, vA, mA0, mA1);
    face(vA, mA0, mA1, gA);
    load(ix0, vA, mA0, mA1);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) carry[c][a][b] = T(0);
    T eA = escale(ix0 - 1);
    for (int s = 0; s <= CXc; s++) {
        step(s, gA, gB, vA, mA0, mA1, eA);
        // the upper face becomes the next lower face (computed values: no wait)
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 2; b++) gA[c][a][b] = gB[c][a][b];
    }
    }  // column segments
    if constexpr (DOT) {
        const double sblk = block_sum<NT>(dot, s_red);
        if (threadIdx.x == 0) epi.dot_partial[blockIdx.x] = sblk;
    }
}

// ---------------------------------------------------------------------------------------
// 3D matvec, FP32, two elements per lane (paired register x-march)
// ---------------------------------------------------------------------------------------
// As k_matvec_h8r, but lane l of a warp computes the two z-neighbouring elements of columns
// ka = kz0 - 1 + 2l and kb = ka + 1, and reads the node columns ka and kb of its two node rows.
// Every value of the element operator is a pair (element ka, element kb) held in one 64-bit
// register pair and computed by the packed FP32 instructions, so one instruction stream
// serves two elements; the z butterfly needs one shuffle per pair (the next lane's column
// ka is this lane's column kb + 1), the z neighbour on the way back one more, and the row
// exchange moves two nodes per lane.  Lane l < 31 owns node columns kb and kb + 1 of row
// je + 1 (lane 31 none: its upper element's z neighbour lies in the next tile), 62 per warp.
// Cube elements (CM 2) only: the element's scale is folded into the seven coefficients.
constexpr int kZTileP = 62;

template <typename TE, int NW, int MINB, int MODE, bool DOT>
__global__ void __launch_bounds__(NW * 32, MINB)
    k_matvec_h8p(int NX, int NY, int NZ, int CXc, const float* __restrict__ u, const TE* __restrict__ E,
                 const uint8_t* __restrict__ mask, const H8Coef<float> cfs, Epi<float> epi) {
    pdl_wait();
    pdl_trigger();
    constexpr int TY = NW - 1, NT = NW * 32;
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ float2 s_q[2][3][NW][32];
    __shared__ double s_red[NW];
    if (epi.skip && *epi.skip) return;
    constexpr int mode = MODE;
    constexpr bool need_b = mode != PF_EPI_STORE, need_x = mode == PF_EPI_JACOBI || mode == PF_EPI_JACOBI_ADD;
    constexpr bool need_xa = mode == PF_EPI_JACOBI_ADD;
    const int nx = NX + 1, ny = NY + 1, nz = NZ + 1;
    const int tid = threadIdx.x, w = tid >> 5, l = tid & 31;
    const int kz0 = blockIdx.x * kZTileP, jy0 = blockIdx.y * TY, ix0 = blockIdx.z * CXc;
    const int je = jy0 - 1 + w;
    const int ka = kz0 - 1 + 2 * l, kb = ka + 1;  // node columns (and element columns) of this lane
    const bool oka = ka >= 0 && ka < nz, okb = kb < nz;  // kb >= kz0 >= 0
    const bool r0 = je >= 0 && je < ny, r1 = je + 1 < ny;
    const bool erow = je >= 0 && je < NY;
    const bool eA = erow && ka >= 0 && ka < NZ;
    const bool eB = l < 31 && erow && kb < NZ;
    const bool own_row = w < TY && je + 1 < ny;
    const bool ownb = own_row && l < 31 && kb < nz;
    const bool ownn = own_row && l < 31 && kb + 1 < nz;
    const int rows = nz * nx;
    const int base0 = rows * je, base1 = base0 + rows;  // node (row, plane 0, column 0)
    const int eplane = NY * NZ;
    const int ebase = je * NZ;
    const bool has_mask = mask != nullptr;
    const float wgt = epi_omega(epi);
    double dot = 0.0;
    H8Coef<F2> cf;
#pragma unroll
    for (int q = 0; q < 7; q++) cf.c[q] = F2(cfs.c[q]);

    // node values of columns ka, kb in rows je, je+1 of plane p (zero outside the mesh)
    auto load = [&](int p, float (&va)[2][3], float (&vb)[2][3], int (&m)[2][2]) {
        const bool pok = p >= 0 && p < nx;
        const int pa0 = base0 + nz * p + ka, pa1 = base1 + nz * p + ka;
        m[0][0] = m[0][1] = m[1][0] = m[1][1] = 0;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            va[0][c] = (pok && r0 && oka) ? u[3 * pa0 + c] : 0.f;
            vb[0][c] = (pok && r0 && okb) ? u[3 * (pa0 + 1) + c] : 0.f;
            va[1][c] = (pok && r1 && oka) ? u[3 * pa1 + c] : 0.f;
            vb[1][c] = (pok && r1 && okb) ? u[3 * (pa1 + 1) + c] : 0.f;
        }
        if (has_mask) {
            if (pok && r0 && oka) m[0][0] = mask[pa0];
            if (pok && r0 && okb) m[0][1] = mask[pa0 + 1];
            if (pok && r1 && oka) m[1][0] = mask[pa1];
            if (pok && r1 && okb) m[1][1] = mask[pa1 + 1];
        }
    };
    // transformed face of both elements: y stage per column, z stage with the pair's upper
    // columns (kb, next lane's ka)
    auto face = [&](float (&va)[2][3], float (&vb)[2][3], const int (&m)[2][2], F2 (&g)[3][2][2]) {
        if (__any_sync(FULL, m[0][0] | m[0][1] | m[1][0] | m[1][1])) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if ((m[0][0] >> c) & 1) va[0][c] = 0.f;
                if ((m[0][1] >> c) & 1) vb[0][c] = 0.f;
                if ((m[1][0] >> c) & 1) va[1][c] = 0.f;
                if ((m[1][1] >> c) & 1) vb[1][c] = 0.f;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const F2 v0(va[0][c], vb[0][c]), v1(va[1][c], vb[1][c]);
            const F2 sm = v1 + v0, df = v1 - v0;
            const float sa_n = __shfl_down_sync(FULL, sm.x(), 1), da_n = __shfl_down_sync(FULL, df.x(), 1);
            const F2 sn(sm.y(), sa_n), dn(df.y(), da_n);
            g[c][0][0] = sm + sn;
            g[c][0][1] = sn - sm;
            g[c][1][0] = df + dn;
            g[c][1][1] = dn - df;
        }
    };
    auto escale = [&](int ie) -> F2 {
        const bool ok = ie >= 0 && ie < NX;
        const int e = ebase + eplane * ie;
        const float a = (ok && eA) ? elem_scale<float>(E[e + ka]) : 0.f;
        const float b = (ok && eB) ? elem_scale<float>(E[e + kb]) : 0.f;
        return F2(a, b);
    };

    F2 carry[3][2][2];
    auto step = [&](int s, F2 (&gl)[3][2][2], F2 (&gh)[3][2][2], float (&va)[2][3], float (&vb)[2][3],
                    int (&m)[2][2], F2& e) {
        const int ie = ix0 - 1 + s;
        face(va, vb, m, gh);
        if (s < CXc) load(ie + 2, va, vb, m);
        const bool out_now = s >= 1 && ie < nx;
        const int nob = base1 + nz * ie + kb;  // owned nodes nob (column kb) and nob + 1
        F2 G[3][2][2];
        h8_element<F2, 2>(gl, gh, e, cf, nullptr, carry, G);
        e = (s < CXc) ? escale(ie + 1) : F2(0.f);
        // epilogue operands of the owned nodes, loaded after the element operator (held
        // across it they would spill), consumed after the barrier
        float pb[2][3], px[2][3], pd[2][3], pa[2][3], pt[2][3];
        int mo[2] = {0, 0};
        if (out_now) {
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const bool own = q == 0 ? ownb : ownn;
                if (!own) continue;
                const int no = nob + q;
                if (has_mask) mo[q] = mask[no];
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    if constexpr (need_b) pb[q][c] = epi.b[3 * no + c];
                    if constexpr (need_x) px[q][c] = epi.x[3 * no + c];
                    if constexpr (need_x) pd[q][c] = epi.dinv[3 * no + c];
                    if constexpr (need_xa) pa[q][c] = epi.xadd[3 * no + c];
                    if constexpr (DOT) pt[q][c] = epi.dot_a[3 * no + c];
                }
            }
        }
        // inverse y and z stages: node kb = (lower element's upper z) + (upper element's lower
        // z); node kb + 1 = (upper element's upper z) + (next lane's lower element's lower z)
        float P1[2][3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const F2 r0a = G[c][0][0] - G[c][1][0], r0b = G[c][0][1] - G[c][1][1];
            const F2 r1a = G[c][0][0] + G[c][1][0], r1b = G[c][0][1] + G[c][1][1];
            const F2 lo0 = r0a - r0b, up0 = r0a + r0b, lo1 = r1a - r1b, up1 = r1a + r1b;
            P1[0][c] = up1.x() + lo1.y();
            P1[1][c] = up1.y() + __shfl_down_sync(FULL, lo1.x(), 1);
            const float q0 = up0.x() + lo0.y();
            const float q1 = up0.y() + __shfl_down_sync(FULL, lo0.x(), 1);
            s_q[s & 1][c][w][l] = make_float2(q0, q1);
        }
        __syncthreads();
        if (out_now) {
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const bool own = q == 0 ? ownb : ownn;
                if (!own) continue;
                const int no = nob + q;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float2 sq = s_q[s & 1][c][w + 1][l];
                    float y = P1[q][c] + (q == 0 ? sq.x : sq.y);
                    if ((mo[q] >> c) & 1) y = u[3 * no + c];
                    float o = y;
                    if constexpr (mode == PF_EPI_RESID) {
                        o = pb[q][c] - y;
                    } else if constexpr (mode == PF_EPI_JACOBI) {
                        o = px[q][c] + wgt * pd[q][c] * (pb[q][c] - y);
                    } else if constexpr (mode == PF_EPI_JACOBI_ADD) {
                        o = pa[q][c] + px[q][c] + wgt * pd[q][c] * (pb[q][c] - y);
                    }
                    epi.out[3 * no + c] = o;
                    if constexpr (DOT) dot += (double)pt[q][c] * (double)(epi.dot_of_y ? y : o);
                }
            }
        }
    };

    F2 gA[3][2][2], gB[3][2][2];
    float vA[2][3], vB[2][3];
    int mk[2][2];
    load(ix0 - 1, vA, vB, mk);
    face(vA, vB, mk, gA);
    load(ix0, vA, vB, mk);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) carry[c][a][b] = F2(0.f);
    F2 eP = escale(ix0 - 1);
    for (int s = 0; s <= CXc; s++) {
        step(s, gA, gB, vA, vB, mk, eP);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int a = 0; a < 2; a++)
#pragma unroll
                for (int b = 0; b < 2; b++) gA[c][a][b] = gB[c][a][b];
    }
    if constexpr (DOT) {
        const double sblk = block_sum<NT>(dot, s_red);
        if (threadIdx.x == 0)
            epi.dot_partial[blockIdx.x + gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z)] = sblk;
    }
}

template <typename T>
static H8Blk<T> make_blk(const Op* op) {
    H8Blk<T> b;
    for (int p = 0; p < 8; p++)
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) b.b[p][i][j] = (T)op->blk[p][i][j];
    return b;
}

// register x-march: NW warps per block (NW - 1 owned node rows), at least MINB blocks per SM
// (FP64: 8 warps x 2 blocks, up to 128 registers; FP32: 12 warps x 2 blocks, up to 80;
// FP32 with 9 warps x 3 blocks at 72 registers measured slower)
constexpr int kNWr64 = 8, kMinBr64 = 2, kNWr32 = 12, kMinBr32 = 2;

// Balanced persistent launch: the (tile column, node plane) work of the grid, node planes
// contiguous within a column, is split evenly over one block per resident slot (at least a
// few planes per block); a block marches its share in at most a few column segments, each
// with one boundary element step.  This avoids both the partial last wave and the
// per-chunk boundary steps of a launch of fixed-length chunks.
static void h8r_launch_dims(const Grid& g, bool fp32, dim3* grid, H8Tiles* tl) {
    const int ny = g.nn[1], nz = g.nn[2], nx = g.nn[0];
    const int nw = fp32 ? kNWr32 : kNWr64;
    const int tz = (nz + kZTileR - 1) / kZTileR;
    const bool half = nz - (tz - 1) * kZTileR <= kZTileR / 2 - 1;
    tl->tzA = half ? tz - 1 : tz;
    tl->tyA = (ny + nw - 2) / (nw - 1);
    const int tyB = half ? (ny + 2 * nw - 2) / (2 * nw - 1) : 0;
    tl->ncols = tl->tzA * tl->tyA + tyB;
    const long long slots = (long long)kNumSM * (fp32 ? kMinBr32 : kMinBr64);
    const long long total = (long long)tl->ncols * nx;
    long long nb = (total + 3) / 4;  // at least four node planes per block
    if (nb > slots) nb = slots;
    if (nb < 1) nb = 1;
    *grid = dim3((unsigned)nb, 1, 1);
}

long long h8_num_blocks(const Grid& g, int fp32) {
    dim3 gr;
    H8Tiles tl;
    h8r_launch_dims(g, fp32 != 0, &gr, &tl);
    return (long long)gr.x * gr.y * gr.z;
}

// paired FP32 kernel: 12 warps (11 owned node rows), 1 block per SM (up to 168 registers:
// at 2 blocks x 8 warps the 128-register cap spilled), 62 owned columns
constexpr int kNWp = 12, kMinBp = 1;
static void h8p_launch_dims(const Grid& g, dim3* grid, int* CXc) {
    const int ny = g.nn[1], nz = g.nn[2], nx = g.nn[0];
    const int tz = (nz + kZTileP - 1) / kZTileP, ty = (ny + kNWp - 2) / (kNWp - 1);
    const long long slots = (long long)kNumSM * kMinBp;
    const long long cols = (long long)tz * ty;
    int best = 4;
    long long best_cost = -1;
    for (int cx = 4; cx <= 64; cx++) {
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
static bool use_paired(const Op* op) { return op->grid.dim == 3 && op->cube && op->variant == 1; }

// ---------------------------------------------------------------------------------------
// 2D matvec (node gather, dense 8x8 K0)
// ---------------------------------------------------------------------------------------
template <typename T>
struct Q4K {
    T k[8][8];
};

template <typename T, typename TE>
__global__ void __launch_bounds__(256) k_matvec_q4(int NX, int NY, const T* __restrict__ u, const TE* __restrict__ E,
                                                   const uint8_t* __restrict__ mask, const Q4K<T> K, Epi<T> epi) {
    pdl_wait();
    pdl_trigger();
    __shared__ double s_red[8];
    if (epi.skip && *epi.skip) return;
    const int nx = NX + 1, ny = NY + 1;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dot = 0.0;
    const T wgt = epi_omega(epi);
    if (n < (long long)nx * ny) {
        const int i = (int)(n % nx), j = (int)(n / nx);
        const uint8_t mn = mask ? mask[n] : (uint8_t)0;
        T acc0 = T(0), acc1 = T(0);
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int ei = i - kCXd(r), ej = j - kCYd(r);
            if (ei < 0 || ej < 0 || ei >= NX || ej >= NY) continue;
            const T we = elem_scale<T>(E[(long long)ei * NY + ej]);
            T a0 = T(0), a1 = T(0);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const long long m = (long long)(ei + kCXd(q)) + (long long)nx * (ej + kCYd(q));
                const uint8_t mm = mask ? mask[m] : (uint8_t)0;
                const T u0 = (mm & 1) ? T(0) : u[2 * m], u1 = (mm & 2) ? T(0) : u[2 * m + 1];
                a0 = fma(K.k[2 * r][2 * q], u0, fma(K.k[2 * r][2 * q + 1], u1, a0));
                a1 = fma(K.k[2 * r + 1][2 * q], u0, fma(K.k[2 * r + 1][2 * q + 1], u1, a1));
            }
            acc0 = fma(a0, we, acc0);
            acc1 = fma(a1, we, acc1);
        }
        T y[2] = {acc0, acc1};
#pragma unroll
        for (int c = 0; c < 2; c++) {
            if (mn & (1 << c)) y[c] = u[2 * n + c];
            const long long g = 2 * n + c;
            const T o = epi_apply(epi, g, y[c], wgt);
            epi.out[g] = o;
            if (epi.dot_partial) dot += (double)epi.dot_a[g] * (double)(epi.dot_of_y ? y[c] : o);
        }
    }
    if (epi.dot_partial) {
        const double sblk = block_sum<256>(dot, s_red);
        if (threadIdx.x == 0) epi.dot_partial[blockIdx.x] = sblk;
    }
}

template <typename T>
static Q4K<T> make_q4k(const Op* op) {
    Q4K<T> K;
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) K.k[i][j] = (T)op->K0[i * 8 + j];
    return K;
}

long long q4_num_blocks(const Grid& g) { return (g.n_nodes + 255) / 256; }

// ---------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------
template <typename T, typename TE, int CM, int MODE, bool DOT>
static int h8r_launch(dim3 grid, H8Tiles tl, const Grid& g, const T* u, const TE* E, const uint8_t* mask,
                      const H8Blk<T>& blk, const H8Coef<T>& cf, const Epi<T>& epi, cudaStream_t st) {
    constexpr int MINB = sizeof(T) == 8 ? kMinBr64 : kMinBr32, NW = sizeof(T) == 8 ? kNWr64 : kNWr32;
    PF_CUDA(launch_pdl(k_matvec_h8r<T, TE, NW, MINB, CM, MODE, DOT>, dim3(grid), dim3(NW * 32), 0, st,
                       g.nel[0], g.nel[1], g.nel[2], tl, u, E, mask, blk, cf, epi));
    return PF_OK;
}

// the epilogue mode and the fused dot are template parameters of the kernel
template <typename T, typename TE, int CM>
static int h8r_dispatch(dim3 grid, H8Tiles tl, const Grid& g, const T* u, const TE* E, const uint8_t* mask,
                        const H8Blk<T>& blk, const H8Coef<T>& cf, const Epi<T>& epi, bool dot, cudaStream_t st) {
#define PF_H8R(M, D) return h8r_launch<T, TE, CM, M, D>(grid, tl, g, u, E, mask, blk, cf, epi, st)
    switch (epi.mode) {
        case PF_EPI_STORE:
            if (dot) PF_H8R(PF_EPI_STORE, true);
            PF_H8R(PF_EPI_STORE, false);
        case PF_EPI_RESID:
            if (dot) PF_H8R(PF_EPI_RESID, true);
            PF_H8R(PF_EPI_RESID, false);
        case PF_EPI_JACOBI:
            if (dot) PF_H8R(PF_EPI_JACOBI, true);
            PF_H8R(PF_EPI_JACOBI, false);
        default:
            if (dot) PF_H8R(PF_EPI_JACOBI_ADD, true);
            PF_H8R(PF_EPI_JACOBI_ADD, false);
    }
#undef PF_H8R
}

template <typename TE, int MODE, bool DOT>
static int h8p_launch(dim3 grid, int cx, const Grid& g, const float* u, const TE* E, const uint8_t* mask,
                      const H8Coef<float>& cf, const Epi<float>& epi, cudaStream_t st) {
    PF_CUDA(launch_pdl(k_matvec_h8p<TE, kNWp, kMinBp, MODE, DOT>, dim3(grid), dim3(kNWp * 32), 0, st, g.nel[0],
                       g.nel[1], g.nel[2], cx, u, E, mask, cf, epi));
    return PF_OK;
}

template <typename TE>
static int h8p_dispatch(const Op* op, const TE* E, const float* u, const uint8_t* mask, const Epi<float>& epi,
                        cudaStream_t st) {
    const Grid& g = op->grid;
    H8Coef<float> cf;
    for (int q = 0; q < 33; q++) cf.c[q] = 0.f;
    const double* v = op->cube_v;
    const double vals[7] = {v[0] - v[1], v[1], v[2], v[3], v[4], v[5] - v[6], v[6]};
    for (int q = 0; q < 7; q++) cf.c[q] = (float)vals[q];
    dim3 grid;
    int cx;
    h8p_launch_dims(g, &grid, &cx);
    pf::count_launch();
    const bool dot = epi.dot_partial != nullptr;
#define PF_H8P(M, D) return h8p_launch<TE, M, D>(grid, cx, g, u, E, mask, cf, epi, st)
    switch (epi.mode) {
        case PF_EPI_STORE:
            if (dot) PF_H8P(PF_EPI_STORE, true);
            PF_H8P(PF_EPI_STORE, false);
        case PF_EPI_RESID:
            if (dot) PF_H8P(PF_EPI_RESID, true);
            PF_H8P(PF_EPI_RESID, false);
        case PF_EPI_JACOBI:
            if (dot) PF_H8P(PF_EPI_JACOBI, true);
            PF_H8P(PF_EPI_JACOBI, false);
        default:
            if (dot) PF_H8P(PF_EPI_JACOBI_ADD, true);
            PF_H8P(PF_EPI_JACOBI_ADD, false);
    }
#undef PF_H8P
}

template <typename T, typename TE>
int launch_fine_matvec(const Op* op, const TE* E, const T* u, const uint8_t* mask, const Epi<T>& epi,
                       cudaStream_t st) {
    const Grid& g = op->grid;
    if constexpr (sizeof(T) == 4) {
        if (use_paired(op)) {
            if (epi.mode < PF_EPI_STORE || epi.mode > PF_EPI_JACOBI_ADD) return fail(PF_BAD_ARG, "unknown epilogue mode");
            const int s = h8p_dispatch<TE>(op, E, u, mask, epi, st);
            if (s) return s;
            PF_LAUNCH_CHECK("fine matvec launch");
            return PF_OK;
        }
    }
    if (g.dim == 3) {
        // a cube element's seven values (a-b, b, c, d, e, f-g, g), the 33 nonzeros of another
        // isotropic box, or (CM 0) the dense class blocks
        const int cm = op->cube ? 2 : (op->sparse ? 1 : 0);
        H8Coef<T> cf;
        for (int q = 0; q < 33; q++) cf.c[q] = T(0);
        if (cm == 2) {
            const double* v = op->cube_v;
            const double vals[7] = {v[0] - v[1], v[1], v[2], v[3], v[4], v[5] - v[6], v[6]};
            for (int q = 0; q < 7; q++) cf.c[q] = (T)vals[q];
        } else if (cm == 1) {
            for (int q = 0; q < 33; q++) cf.c[q] = (T)op->coef[q];
        }
        const H8Blk<T> blk = make_blk<T>(op);
        if (epi.mode < PF_EPI_STORE || epi.mode > PF_EPI_JACOBI_ADD) return fail(PF_BAD_ARG, "unknown epilogue mode");
        dim3 grid;
        H8Tiles tl;
        h8r_launch_dims(g, sizeof(T) == 4, &grid, &tl);
        pf::count_launch();
        const bool dot = epi.dot_partial != nullptr;
        int s;
        if (cm == 2)
            s = h8r_dispatch<T, TE, 2>(grid, tl, g, u, E, mask, blk, cf, epi, dot, st);
        else if (cm == 1)
            s = h8r_dispatch<T, TE, 1>(grid, tl, g, u, E, mask, blk, cf, epi, dot, st);
        else
            s = h8r_dispatch<T, TE, 0>(grid, tl, g, u, E, mask, blk, cf, epi, dot, st);
        if (s) return s;
    } else {
        const long long nb = q4_num_blocks(g);
        pf::count_launch();
        PF_CUDA(launch_pdl(k_matvec_q4<T, TE>, dim3((unsigned)nb), dim3(256), 0, st, g.nel[0], g.nel[1], u, E, mask, make_q4k<T>(op), epi));
    }
    PF_LAUNCH_CHECK("fine matvec launch");
    return PF_OK;
}

long long fine_matvec_num_blocks(const Op* op, int fp32) {
    if (fp32 && use_paired(op)) {
        dim3 gr;
        int cx;
        h8p_launch_dims(op->grid, &gr, &cx);
        return (long long)gr.x * gr.y * gr.z;
    }
    return op->grid.dim == 3 ? h8_num_blocks(op->grid, fp32) : q4_num_blocks(op->grid);
}

template int launch_fine_matvec<double, double>(const Op*, const double*, const double*, const uint8_t*,
                                                const Epi<double>&, cudaStream_t);
template int launch_fine_matvec<float, float>(const Op*, const float*, const float*, const uint8_t*,
                                              const Epi<float>&, cudaStream_t);
template int launch_fine_matvec<float, __nv_bfloat16>(const Op*, const __nv_bfloat16*, const float*, const uint8_t*,
                                                      const Epi<float>&, cudaStream_t);

// ---------------------------------------------------------------------------------------
// diagonal, sensitivity, mask packing
// ---------------------------------------------------------------------------------------
struct KDiag {
    double d[24];
};

template <typename T>
__global__ void k_diagonal(Grid g, const double* __restrict__ E, const uint8_t* __restrict__ mask, KDiag kd,
                           T* __restrict__ diag) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.n_nodes) return;
    const int dof = g.dim, nc = g.dim == 3 ? 8 : 4;
    int i, j, k;
    const unsigned un = (unsigned)n;  // fewer than 2^31 nodes (validate_grid)
    if (g.dim == 3) {
        const unsigned t = un / (unsigned)g.nn[2];
        k = (int)(un - t * (unsigned)g.nn[2]);
        j = (int)(t / (unsigned)g.nn[0]);
        i = (int)(t - (unsigned)j * (unsigned)g.nn[0]);
    } else {
        j = (int)(un / (unsigned)g.nn[0]);
        i = (int)(un - (unsigned)j * (unsigned)g.nn[0]);
        k = 0;
    }
    const uint8_t m = mask ? mask[n] : (uint8_t)0;
    double s[3] = {0, 0, 0};
    for (int r = 0; r < nc; r++) {
        const int ei = i - kCXd(r), ej = j - kCYd(r), ek = g.dim == 3 ? k - kCZd(r) : 0;
        if (ei < 0 || ej < 0 || ei >= g.nel[0] || ej >= g.nel[1]) continue;
        if (g.dim == 3 && (ek < 0 || ek >= g.nel[2])) continue;
        const long long e = g.dim == 3 ? ((long long)ei * g.nel[1] + ej) * g.nel[2] + ek : (long long)ei * g.nel[1] + ej;
        const double we = E[e];
        for (int d = 0; d < dof; d++) s[d] += kd.d[r * dof + d] * we;
    }
    for (int d = 0; d < dof; d++) diag[n * dof + d] = (m & (1 << d)) ? T(1) : (T)s[d];
}

template <typename T>
int launch_diagonal(const Op* op, const double* E, const uint8_t* mask, T* diag, cudaStream_t st) {
    const Grid& g = op->grid;
    KDiag kd;
    const int nd = (g.dim == 3 ? 8 : 4) * g.dim;
    for (int i = 0; i < nd; i++) kd.d[i] = op->K0[i * nd + i];
    pf::count_launch();
    k_diagonal<T><<<(unsigned)((g.n_nodes + 255) / 256), 256, 0, st>>>(g, E, mask, kd, diag);
    PF_LAUNCH_CHECK("diagonal launch");
    return PF_OK;
}
template int launch_diagonal<double>(const Op*, const double*, const uint8_t*, double*, cudaStream_t);
template int launch_diagonal<float>(const Op*, const double*, const uint8_t*, float*, cudaStream_t);

// Element energy e_e = u_e^T K0 u_e = (T u_e)^T B (T u_e) (H8, Walsh basis) or the dense
// quadratic form (Q4).  ADJ = false: dk_e = -e_e (reference process_dk, grad.cu:1-16).
// ADJ = true (the fused adjoint of the compliance): out_e = scale * dE/drho(rho_e) * (-e_e)
// with the SIMP derivative of the reference's penalize_grad
// (Problem/CUDA/MinimumCompliance.py:351-367), i.e. the element factor of
// dc/dx = H^T [dE/drho * (-u_e^T K0 u_e)] before the filter transpose.
struct AdjArgs {
    const double* rho;
    pf_simp_params P;
    double scale;
};

__device__ __forceinline__ double simp_grad(double r, const pf_simp_params& P) {
    double dh = 1.0;
    if (P.heavyside) {
        const double den = tanh(P.beta * P.eta) + tanh(P.beta * (1.0 - P.eta));
        const double t = tanh(P.beta * (r - P.eta));
        r = (tanh(P.beta * P.eta) + t) / den;
        dh = P.beta * (1.0 - t * t) / den;
    }
    return P.penalty * pow(r, P.penalty - 1.0) * dh * P.E_mul;
}

template <bool ADJ>
__global__ void k_sens_h8(int NX, int NY, int NZ, const double* __restrict__ U, const H8Blk<double> blk,
                          AdjArgs adj, double* __restrict__ dk) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)NX * NY * NZ) return;
    const int k = (int)(e % NZ), j = (int)((e / NZ) % NY), i = (int)(e / ((long long)NY * NZ));
    const int nx = NX + 1, nz = NZ + 1;
    double v[3][2][2][2];  // [comp][a][b][c] corner values -> Walsh coefficients in place
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const long long n = (long long)(k + c) + (long long)nz * ((i + a) + (long long)nx * (j + b));
#pragma unroll
                for (int d = 0; d < 3; d++) v[d][a][b][c] = U[3 * n + d];
            }
#pragma unroll
    for (int d = 0; d < 3; d++) {
#pragma unroll
        for (int b = 0; b < 2; b++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const double x0 = v[d][0][b][c], x1 = v[d][1][b][c];
                v[d][0][b][c] = x0 + x1;
                v[d][1][b][c] = x1 - x0;
            }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const double x0 = v[d][a][0][c], x1 = v[d][a][1][c];
                v[d][a][0][c] = x0 + x1;
                v[d][a][1][c] = x1 - x0;
            }
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const double x0 = v[d][a][b][0], x1 = v[d][a][b][1];
                v[d][a][b][0] = x0 + x1;
                v[d][a][b][1] = x1 - x0;
            }
    }
    double q = 0.0;
#pragma unroll
    for (int p = 0; p < 8; p++) {
        const int px = p & 1, py = (p >> 1) & 1, pz = (p >> 2) & 1;
        const double i0 = v[0][px ^ 1][py][pz], i1 = v[1][px][py ^ 1][pz], i2 = v[2][px][py][pz ^ 1];
        const double o0 = blk.b[p][0][0] * i0 + blk.b[p][0][1] * i1 + blk.b[p][0][2] * i2;
        const double o1 = blk.b[p][1][0] * i0 + blk.b[p][1][1] * i1 + blk.b[p][1][2] * i2;
        const double o2 = blk.b[p][2][0] * i0 + blk.b[p][2][1] * i1 + blk.b[p][2][2] * i2;
        q += i0 * o0 + i1 * o1 + i2 * o2;
    }
    if (ADJ)
        dk[e] = adj.scale * simp_grad(adj.rho[e], adj.P) * (-q);
    else
        dk[e] = -q;
}

template <bool ADJ>
__global__ void k_sens_q4(int NX, int NY, const double* __restrict__ U, const Q4K<double> K, AdjArgs adj,
                          double* __restrict__ dk) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)NX * NY) return;
    const int i = (int)(e / NY), j = (int)(e % NY), nx = NX + 1;
    double ue[8];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const long long m = (long long)(i + kCXd(q)) + (long long)nx * (j + kCYd(q));
        ue[2 * q] = U[2 * m];
        ue[2 * q + 1] = U[2 * m + 1];
    }
    double out = 0.0;
#pragma unroll
    for (int a = 0; a < 8; a++) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < 8; b++) s += K.k[a][b] * ue[b];
        out -= s * ue[a];
    }
    if (ADJ)
        dk[e] = adj.scale * simp_grad(adj.rho[e], adj.P) * out;
    else
        dk[e] = out;
}

template <bool ADJ>
static int launch_sens(const Op* op, const double* U, const AdjArgs& adj, double* out, cudaStream_t st) {
    const Grid& g = op->grid;
    const unsigned nb = (unsigned)((g.n_elem + 255) / 256);
    pf::count_launch();
    if (g.dim == 3)
        k_sens_h8<ADJ><<<nb, 256, 0, st>>>(g.nel[0], g.nel[1], g.nel[2], U, make_blk<double>(op), adj, out);
    else
        k_sens_q4<ADJ><<<nb, 256, 0, st>>>(g.nel[0], g.nel[1], U, make_q4k<double>(op), adj, out);
    PF_LAUNCH_CHECK("sensitivity launch");
    return PF_OK;
}

int launch_sensitivity(const Op* op, const double* U, double* dk, cudaStream_t st) {
    AdjArgs none;
    memset(&none, 0, sizeof(none));
    return launch_sens<false>(op, U, none, dk, st);
}

int launch_adjoint(const Op* op, const double* U, const double* rho, const pf_simp_params& P, double scale,
                   double* out, cudaStream_t st) {
    AdjArgs a;
    a.rho = rho;
    a.P = P;
    a.scale = scale;
    return launch_sens<true>(op, U, a, out, st);
}

__global__ void k_pack_mask(long long n_nodes, int dof, const uint8_t* __restrict__ con, uint8_t* __restrict__ mask) {
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nodes) return;
    uint8_t m = 0;
    for (int d = 0; d < dof; d++)
        if (con[n * dof + d]) m |= (uint8_t)(1 << d);
    mask[n] = m;
}

int launch_pack_mask(const Op* op, const uint8_t* con, uint8_t* mask, cudaStream_t st) {
    const Grid& g = op->grid;
    pf::count_launch();
    k_pack_mask<<<(unsigned)((g.n_nodes + 255) / 256), 256, 0, st>>>(g.n_nodes, g.dof, con, mask);
    PF_LAUNCH_CHECK("pack mask launch");
    return PF_OK;
}

}  // namespace pf
