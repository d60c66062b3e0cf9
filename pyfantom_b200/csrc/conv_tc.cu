// 3x3x3 convolution (forward, input gradient, weight gradient) on the tensor cores:
// implicit GEMM with tcgen05.mma, BF16 operands staged in shared memory from the FP32
// tensors, FP32 accumulation in tensor memory.
//
//   forward     D[o, co] = sum_k A[o, k] B[k, co],  k = ci*27 + t,
//               A[o, k] = x[n, ci, s*o + t - 1] (zero outside), B[k, co] = w[co, ci, t]
//               y[n, co, o] = D[o, co] + b[co] (ReLU optional)
//   input grad  D[v, ci] = sum_k A[v, k] B[k, ci],  k = co*27 + t,
//               A[v, k] = dy[n, co, (v - t + 1) / s] (where divisible and inside), B[k, ci] = w[co, ci, t]
//               dx[n, ci, v] = D[v, ci] (+= with accumulate)
//   weight grad D[m, co] = sum_k A[m, k] B[co, k] over k = (n, o), m = ci*27 + t plus a row of
//               ones (the bias gradient): A[m, k] = x[n, ci, s*o + t - 1], B[co, k] = dy[n, co, o]
// Layouts are those of the FP32 kernels (cnn.cu): [N][C][X][Y][Z], weights [Cout][Cin][27].
//
// One CTA of 128 threads computes 128 rows (voxels, or weight-gradient rows) against all
// columns (channels, padded to NP, a multiple of 16).  The reduction runs in chunks of 64:
// each thread gathers its row's 64 operands (8 x 16 bytes of BF16) into the canonical
// no-swizzle K-major layout (core matrices of 8 rows x 16 bytes), the threads stage the
// other operand's slice, and one thread issues four 128 x NP x 16 MMAs and commits them to
// the buffer's mbarrier.  Two buffers alternate, so the gather of chunk c+1 overlaps the
// MMAs of chunk c.  After the last chunk each warp reads its 32 rows of the accumulator
// (tcgen05.ld 32x32b) and stores them column by column (32 consecutive rows per store).
// Every wait on an mbarrier is bounded: past the limit the kernel records an error in
// `err`, skips the epilogue, and releases its tensor memory.
#include <cuda_bf16.h>

#include <cstdint>

#include "common.cuh"

#if __has_include(<cute/arch/mma_sm100_desc.hpp>)
#include <cute/arch/mma_sm100_desc.hpp>
#define PF_HAVE_CUTE_DESC 1
#endif

namespace pf {

constexpr int kTcRows = 128;   // rows per CTA (MMA M)
constexpr int kTcKC = 64;      // reduction chunk (4 MMAs of K = 16)
constexpr int kTcThreads = 128;
constexpr long long kTcSpin = 1LL << 20;  // try_wait polls before giving up

// ---- descriptors -----------------------------------------------------------------------
// shared-memory matrix descriptor, K-major, no swizzle: start address, leading byte offset
// (between the two 8-element K halves of a 16-wide slice), stride byte offset (between
// 8-row groups), all in 16-byte units; version 1 (sm_100).
__host__ __device__ constexpr uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator, M x N
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4)                       // D format F32
           | (1u << 7) | (1u << 10)        // A, B format BF16
           | ((uint32_t)(N >> 3) << 17)    // N / 8
           | ((uint32_t)(M >> 4) << 24);   // M / 16
}

// The encodings above against CuTe's bit-field definitions of the same descriptors (when
// its headers are on the include path): checked once on the host before the first launch.
static bool tc_encodings_match() {
#ifdef PF_HAVE_CUTE_DESC
    const uint32_t i64 = uint32_t(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 64,
                                                              cute::UMMA::Major::K, cute::UMMA::Major::K>());
    const uint32_t i16 = uint32_t(cute::UMMA::make_instr_desc<cute::bfloat16_t, cute::bfloat16_t, float, 128, 16,
                                                              cute::UMMA::Major::K, cute::UMMA::Major::K>());
    cute::UMMA::SmemDescriptor d;
    d.desc_ = 0;
    d.start_address_ = (uint16_t)(0x1230 >> 4);
    d.leading_byte_offset_ = (uint16_t)(2048 >> 4);
    d.stride_byte_offset_ = (uint16_t)(128 >> 4);
    d.version_ = 1;
    d.lbo_mode_ = 0;
    d.base_offset_ = 0;
    d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_NONE);
    return i64 == umma_idesc_bf16(128, 64) && i16 == umma_idesc_bf16(128, 16) &&
           uint64_t(d) == umma_smem_desc(0x1230, 2048, 128);
#else
    return true;
#endif
}

// ---- PTX wrappers ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long long i = 0; i < kTcSpin; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tc_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&h);
}

struct ConvTcArgs {
    const float* src;  // forward, weight grad: x; input gradient: dy
    const float* w;    // forward, input gradient: weights; weight grad: dy
    const float* b;    // forward bias
    float* dst;        // forward: y, input gradient: dx
    int* err;
    int N, Cin, Cout, s, relu, accumulate;
    int X, Y, Z, Xo, Yo, Zo;
};

// shared memory of one CTA: A0 A1 (rows x chunk) B0 B1 (NP x chunk), 2 mbarriers, TMEM slot
__device__ __forceinline__ size_t tc_a_bytes() { return (size_t)kTcRows * kTcKC * 2; }
static size_t tc_smem_bytes(int NP) {
    return 2 * ((size_t)kTcRows * kTcKC * 2 + (size_t)NP * kTcKC * 2) + 2 * sizeof(uint64_t) + 16;
}

// Stage 8 consecutive-k values of row `row` of A (rows x 64 chunk) at group g, and the MMA
// issue/commit of one chunk: shared by the three kernels.
__device__ __forceinline__ void tc_store_a(uint8_t* sA, int row, int g, uint4 q) {
    const int slice = g >> 1, half = g & 1;
    *reinterpret_cast<uint4*>(sA + slice * (kTcRows * 32) + half * (kTcRows * 16) + (row >> 3) * 128 + (row & 7) * 16) = q;
}
__device__ __forceinline__ void tc_store_b(uint8_t* sB, int NP, int j, int g, uint4 q) {
    const int slice = g >> 1, half = g & 1;
    *reinterpret_cast<uint4*>(sB + slice * (NP * 32) + half * (NP * 16) + (j >> 3) * 128 + (j & 7) * 16) = q;
}
__device__ __forceinline__ void tc_issue_chunk(uint32_t tmem, const uint8_t* sA, const uint8_t* sB, int NP,
                                               uint32_t idesc, long long k0, long long kend, bool first,
                                               uint64_t* bar) {
    tc_fence_after();
    const uint32_t abase = smem_u32(sA), bbase = smem_u32(sB);
#pragma unroll
    for (int j = 0; j < kTcKC / 16; j++) {
        if (k0 + j * 16 >= kend) break;
        const uint64_t da = umma_smem_desc(abase + j * (kTcRows * 32), kTcRows * 16, 128);
        const uint64_t db = umma_smem_desc(bbase + j * (NP * 32), NP * 16, 128);
        tc_mma(tmem, da, db, idesc, (!first || j > 0) ? 1u : 0u);
    }
    tc_commit(bar);
}
__device__ __forceinline__ uint32_t tc_setup(uint8_t* smem, int NP, int ncols, uint64_t** bars_out) {
    const int tid = threadIdx.x, warp = tid >> 5;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * (tc_a_bytes() + (size_t)NP * kTcKC * 2));
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
    if (warp == 0) {
        tc_alloc(tslot, (uint32_t)ncols);
        tc_relinquish();
    }
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    *bars_out = bars;
    return *tslot;
}

// MODE 0: forward, MODE 1: input gradient
template <int MODE>
__global__ void __launch_bounds__(kTcThreads, 1) k_conv_tc(ConvTcArgs a, int NP, int ncols) {
    extern __shared__ __align__(128) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    // rows: output voxels (forward) or input voxels (input gradient)
    const int RX = MODE == 0 ? a.Xo : a.X, RY = MODE == 0 ? a.Yo : a.Y, RZ = MODE == 0 ? a.Zo : a.Z;
    const long long Vr = (long long)RX * RY * RZ;
    const int NCH = MODE == 0 ? a.Cout : a.Cin;  // GEMM columns (output channels of the product)
    const int KCH = MODE == 0 ? a.Cin : a.Cout;  // reduction channels
    const int K = KCH * 27;
    const int nchunks = (K + kTcKC - 1) / kTcKC;
    const int n = blockIdx.y;
    const size_t a_bytes = tc_a_bytes(), b_bytes = (size_t)NP * kTcKC * 2;
    auto sA = [&](int buf) { return smem + buf * a_bytes; };
    auto sB = [&](int buf) { return smem + 2 * a_bytes + buf * b_bytes; };
    uint64_t* bars;
    const uint32_t tmem = tc_setup(smem, NP, ncols, &bars);

    const long long r = (long long)blockIdx.x * kTcRows + tid;
    const bool rv = r < Vr;
    int rx = 0, ry = 0, rz = 0;
    if (rv) {
        rz = (int)(r % RZ);
        ry = (int)((r / RZ) % RY);
        rx = (int)(r / ((long long)RZ * RY));
    }
    const float* src_n =
        a.src + (long long)n * KCH * (MODE == 0 ? (long long)a.X * a.Y * a.Z : (long long)a.Xo * a.Yo * a.Zo);
    const uint32_t idesc = umma_idesc_bf16(kTcRows, NP);

    // operand A[r, k] of this thread's row
    auto a_val = [&](int k) -> float {
        if (!rv || k >= K) return 0.f;
        const int c = k / 27, t = k - c * 27;
        const int tx = t / 9, ty = (t / 3) % 3, tz = t % 3;
        if constexpr (MODE == 0) {
            const int ix = a.s * rx + tx - 1, iy = a.s * ry + ty - 1, iz = a.s * rz + tz - 1;
            if (ix < 0 || iy < 0 || iz < 0 || ix >= a.X || iy >= a.Y || iz >= a.Z) return 0.f;
            return __ldg(src_n + (((long long)c * a.X + ix) * a.Y + iy) * a.Z + iz);
        } else {
            const int px = rx - tx + 1, py = ry - ty + 1, pz = rz - tz + 1;
            if (px < 0 || py < 0 || pz < 0 || px % a.s || py % a.s || pz % a.s) return 0.f;
            const int ox = px / a.s, oy = py / a.s, oz = pz / a.s;
            if (ox >= a.Xo || oy >= a.Yo || oz >= a.Zo) return 0.f;
            return __ldg(src_n + (((long long)c * a.Xo + ox) * a.Yo + oy) * a.Zo + oz);
        }
    };
    // operand B[k, j] (j an output channel of the product)
    auto b_val = [&](int j, int k) -> float {
        if (j >= NCH || k >= K) return 0.f;
        if constexpr (MODE == 0) {
            return __ldg(a.w + (long long)j * K + k);
        } else {
            const int co = k / 27, t = k - co * 27;
            return __ldg(a.w + ((long long)co * a.Cin + j) * 27 + t);
        }
    };

    bool ok = true;
    uint32_t phases = 0u;  // bit b: parity of the next completion of buffer b's barrier
    for (int c = 0; c < nchunks; c++) {
        const int buf = c & 1;
        if (c >= 2) {  // the MMAs of chunk c - 2 read this buffer
            if (!mbar_wait(&bars[buf], (phases >> buf) & 1u)) ok = false;
            phases ^= 1u << buf;
        }
        const int k0 = c * kTcKC;
#pragma unroll 1
        for (int g = 0; g < kTcKC / 8; g++) {
            const int kb = k0 + g * 8;
            uint4 q;
            q.x = pack_bf16(a_val(kb + 0), a_val(kb + 1));
            q.y = pack_bf16(a_val(kb + 2), a_val(kb + 3));
            q.z = pack_bf16(a_val(kb + 4), a_val(kb + 5));
            q.w = pack_bf16(a_val(kb + 6), a_val(kb + 7));
            tc_store_a(sA(buf), tid, g, q);
        }
        for (int idx = tid; idx < NP * (kTcKC / 8); idx += kTcThreads) {
            const int j = idx / (kTcKC / 8), g = idx % (kTcKC / 8);
            const int kb = k0 + g * 8;
            uint4 q;
            q.x = pack_bf16(b_val(j, kb + 0), b_val(j, kb + 1));
            q.y = pack_bf16(b_val(j, kb + 2), b_val(j, kb + 3));
            q.z = pack_bf16(b_val(j, kb + 4), b_val(j, kb + 5));
            q.w = pack_bf16(b_val(j, kb + 6), b_val(j, kb + 7));
            tc_store_b(sB(buf), NP, j, g, q);
        }
        fence_async_smem();  // the generic-proxy stores become visible to the tensor cores
        __syncthreads();
        if (tid == 0) tc_issue_chunk(tmem, sA(buf), sB(buf), NP, idesc, k0, K, c == 0, &bars[buf]);
    }
    // the last commit tracks every MMA issued before it
    const int lb = (nchunks - 1) & 1;
    if (!mbar_wait(&bars[lb], (phases >> lb) & 1u)) ok = false;
    tc_fence_after();
    // tcgen05.ld is warp-collective: decide the epilogue for the whole block
    if (__syncthreads_and(ok ? 1 : 0)) {
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < NP; c0 += 16) {
            float v[16];
            tc_ld16(trow + (uint32_t)c0, v);
            if (rv) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int ch = c0 + i;
                    if (ch >= NCH) break;
                    float* d = a.dst + ((long long)n * NCH + ch) * Vr + r;
                    if constexpr (MODE == 0) {
                        float yv = v[i] + __ldg(a.b + ch);
                        if (a.relu) yv = fmaxf(yv, 0.f);
                        *d = yv;
                    } else {
                        *d = a.accumulate ? *d + v[i] : v[i];
                    }
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(a.err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, (uint32_t)ncols);
}

// Weight gradient: the voxels are split into ranges of kTcWSplit; CTA (row tile, range)
// writes its partial D to part[range][co][m] and k_conv_tc_wsum adds the ranges in order.
constexpr int kTcWSplit = 4096;

__global__ void __launch_bounds__(kTcThreads, 1) k_conv_tc_wgrad(ConvTcArgs a, int NP, int ncols, int Mtot,
                                                                 float* __restrict__ part) {
    extern __shared__ __align__(128) uint8_t smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const long long Vo = (long long)a.Xo * a.Yo * a.Zo, Vi = (long long)a.X * a.Y * a.Z;
    const long long Ktot = (long long)a.N * Vo;
    const long long kbeg = (long long)blockIdx.y * kTcWSplit;
    const long long kend = kbeg + kTcWSplit < Ktot ? kbeg + kTcWSplit : Ktot;
    const int nchunks = (int)((kend - kbeg + kTcKC - 1) / kTcKC);
    const size_t a_bytes = tc_a_bytes(), b_bytes = (size_t)NP * kTcKC * 2;
    auto sA = [&](int buf) { return smem + buf * a_bytes; };
    auto sB = [&](int buf) { return smem + 2 * a_bytes + buf * b_bytes; };
    uint64_t* bars;
    const uint32_t tmem = tc_setup(smem, NP, ncols, &bars);
    // this thread's row: (ci, tap), the bias row, or padding
    const int m = blockIdx.x * kTcRows + tid;
    const int M = 27 * a.Cin;
    const bool is_w = m < M, is_b = m == M;
    const int ci = is_w ? m / 27 : 0, t = is_w ? m % 27 : 0;
    const int tx = t / 9, ty = (t / 3) % 3, tz = t % 3;
    const uint32_t idesc = umma_idesc_bf16(kTcRows, NP);

    auto a_val = [&](long long k) -> float {
        if (k >= kend || !(is_w || is_b)) return 0.f;
        if (is_b) return 1.f;
        const int n = (int)(k / Vo);
        const long long o = k - (long long)n * Vo;
        const int oz = (int)(o % a.Zo), oy = (int)((o / a.Zo) % a.Yo), ox = (int)(o / ((long long)a.Zo * a.Yo));
        const int ix = a.s * ox + tx - 1, iy = a.s * oy + ty - 1, iz = a.s * oz + tz - 1;
        if (ix < 0 || iy < 0 || iz < 0 || ix >= a.X || iy >= a.Y || iz >= a.Z) return 0.f;
        return __ldg(a.src + ((long long)n * a.Cin + ci) * Vi + ((long long)ix * a.Y + iy) * a.Z + iz);
    };
    auto b_val = [&](int co, long long k) -> float {
        if (co >= a.Cout || k >= kend) return 0.f;
        const int n = (int)(k / Vo);
        const long long o = k - (long long)n * Vo;
        return __ldg(a.w + ((long long)n * a.Cout + co) * Vo + o);  // dy
    };

    bool ok = true;
    uint32_t phases = 0u;
    for (int c = 0; c < nchunks; c++) {
        const int buf = c & 1;
        if (c >= 2) {
            if (!mbar_wait(&bars[buf], (phases >> buf) & 1u)) ok = false;
            phases ^= 1u << buf;
        }
        const long long k0 = kbeg + (long long)c * kTcKC;
#pragma unroll 1
        for (int g = 0; g < kTcKC / 8; g++) {
            const long long kb = k0 + g * 8;
            uint4 q;
            q.x = pack_bf16(a_val(kb + 0), a_val(kb + 1));
            q.y = pack_bf16(a_val(kb + 2), a_val(kb + 3));
            q.z = pack_bf16(a_val(kb + 4), a_val(kb + 5));
            q.w = pack_bf16(a_val(kb + 6), a_val(kb + 7));
            tc_store_a(sA(buf), tid, g, q);
        }
        for (int idx = tid; idx < NP * (kTcKC / 8); idx += kTcThreads) {
            const int j = idx / (kTcKC / 8), g = idx % (kTcKC / 8);
            const long long kb = k0 + g * 8;
            uint4 q;
            q.x = pack_bf16(b_val(j, kb + 0), b_val(j, kb + 1));
            q.y = pack_bf16(b_val(j, kb + 2), b_val(j, kb + 3));
            q.z = pack_bf16(b_val(j, kb + 4), b_val(j, kb + 5));
            q.w = pack_bf16(b_val(j, kb + 6), b_val(j, kb + 7));
            tc_store_b(sB(buf), NP, j, g, q);
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) tc_issue_chunk(tmem, sA(buf), sB(buf), NP, idesc, k0, kend, c == 0, &bars[buf]);
    }
    const int lb = (nchunks - 1) & 1;
    if (!mbar_wait(&bars[lb], (phases >> lb) & 1u)) ok = false;
    tc_fence_after();
    if (__syncthreads_and(ok ? 1 : 0)) {
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < NP; c0 += 16) {
            float v[16];
            tc_ld16(trow + (uint32_t)c0, v);
            if (m < Mtot) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const int co = c0 + i;
                    if (co >= a.Cout) break;
                    part[((long long)blockIdx.y * a.Cout + co) * Mtot + m] = v[i];
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(a.err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tc_dealloc(tmem, (uint32_t)ncols);
}

// dw[co, ci, t] = sum over ranges of part[range][co][ci*27 + t]; db[co] from the ones row
__global__ void k_conv_tc_wsum(const float* __restrict__ part, int nsplit, int Cout, int Mtot, float* __restrict__ dw,
                               float* __restrict__ db) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)Cout * Mtot) return;
    const int co = (int)(i / Mtot), m = (int)(i - (long long)co * Mtot);
    float s = 0.f;
    for (int r = 0; r < nsplit; r++) s += part[((long long)r * Cout + co) * Mtot + m];
    if (m < Mtot - 1)
        dw[(long long)co * (Mtot - 1) + m] = s;
    else if (db)
        db[co] = s;
}

static int tc_ncols(int NP) {
    int c = 32;
    while (c < NP) c <<= 1;
    return c;
}

static int tc_check(int NP) {
    if (NP > 256) return fail(PF_UNSUPPORTED, "tensor-core conv: at most 256 output channels");
    static const bool enc_ok = tc_encodings_match();
    if (!enc_ok) return fail(PF_UNSUPPORTED, "tensor-core conv: descriptor encoding check failed");
    return PF_OK;
}

template <int MODE>
static int launch_conv_tc(const ConvTcArgs& a, cudaStream_t st) {
    const int NCH = MODE == 0 ? a.Cout : a.Cin;
    const int NP = (NCH + 15) / 16 * 16;
    int s = tc_check(NP);
    if (s) return s;
    const long long Vr = MODE == 0 ? (long long)a.Xo * a.Yo * a.Zo : (long long)a.X * a.Y * a.Z;
    const size_t smem = tc_smem_bytes(NP);
    PF_CUDA(cudaFuncSetAttribute(k_conv_tc<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((Vr + kTcRows - 1) / kTcRows), (unsigned)a.N);
    pf::count_launch();
    k_conv_tc<MODE><<<grid, kTcThreads, smem, st>>>(a, NP, tc_ncols(NP));
    PF_LAUNCH_CHECK("tensor-core conv launch");
    return PF_OK;
}

static inline int out_ext(int n, int s) { return (n - 1) / s + 1; }

}  // namespace pf

using namespace pf;

extern "C" int pf_cnn_conv3d_fwd_tc(const float* x, int N, int Cin, int X, int Y, int Z, const float* w, const float* b,
                                    int Cout, int stride, int relu, float* y, int* err, void* stream) {
    if (!x || !w || !b || !y || !err || N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 ||
        (stride != 1 && stride != 2))
        return fail(PF_BAD_ARG, "pf_cnn_conv3d_fwd_tc: bad argument");
    ConvTcArgs a = {x, w, b, y, err, N, Cin, Cout, stride, relu, 0, X, Y, Z,
                    out_ext(X, stride), out_ext(Y, stride), out_ext(Z, stride)};
    return launch_conv_tc<0>(a, as_stream(stream));
}

extern "C" int pf_cnn_conv3d_bwd_data_tc(const float* dy, int N, int Cin, int X, int Y, int Z, const float* w,
                                         int Cout, int stride, int accumulate, float* dx, int* err, void* stream) {
    if (!dy || !w || !dx || !err || N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 ||
        (stride != 1 && stride != 2))
        return fail(PF_BAD_ARG, "pf_cnn_conv3d_bwd_data_tc: bad argument");
    ConvTcArgs a = {dy, w, nullptr, dx, err, N, Cin, Cout, stride, 0, accumulate, X, Y, Z,
                    out_ext(X, stride), out_ext(Y, stride), out_ext(Z, stride)};
    return launch_conv_tc<1>(a, as_stream(stream));
}

extern "C" size_t pf_cnn_conv3d_bwd_weight_tc_workspace(int N, int Cin, int X, int Y, int Z, int Cout, int stride) {
    if (N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 || (stride != 1 && stride != 2)) return 0;
    const long long Ktot = (long long)N * out_ext(X, stride) * out_ext(Y, stride) * out_ext(Z, stride);
    const long long nsplit = (Ktot + kTcWSplit - 1) / kTcWSplit;
    return (size_t)(nsplit * Cout * (27LL * Cin + 1));
}

extern "C" int pf_cnn_conv3d_bwd_weight_tc(const float* x, const float* dy, int N, int Cin, int X, int Y, int Z,
                                           int Cout, int stride, float* dw, float* db, float* work, int* err,
                                           void* stream) {
    if (!x || !dy || !dw || !work || !err || N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 ||
        (stride != 1 && stride != 2))
        return fail(PF_BAD_ARG, "pf_cnn_conv3d_bwd_weight_tc: bad argument");
    const int NP = (Cout + 15) / 16 * 16;
    int s = tc_check(NP);
    if (s) return s;
    ConvTcArgs a = {x, dy, nullptr, dw, err, N, Cin, Cout, stride, 0, 0, X, Y, Z,
                    out_ext(X, stride), out_ext(Y, stride), out_ext(Z, stride)};
    const long long Ktot = (long long)N * a.Xo * a.Yo * a.Zo;
    const int nsplit = (int)((Ktot + kTcWSplit - 1) / kTcWSplit);
    const int Mtot = 27 * Cin + 1;
    const size_t smem = tc_smem_bytes(NP);
    cudaStream_t st = as_stream(stream);
    PF_CUDA(cudaFuncSetAttribute(k_conv_tc_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    pf::count_launch(2);
    k_conv_tc_wgrad<<<dim3((unsigned)((Mtot + kTcRows - 1) / kTcRows), (unsigned)nsplit), kTcThreads, smem, st>>>(
        a, NP, tc_ncols(NP), Mtot, work);
    const long long nt = (long long)Cout * Mtot;
    k_conv_tc_wsum<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(work, nsplit, Cout, Mtot, dw, db);
    PF_LAUNCH_CHECK("tensor-core conv weight gradient launch");
    return PF_OK;
}
