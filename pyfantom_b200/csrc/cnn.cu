// Kernels of the learned warm start: a small 3D convolutional network on a cell grid.
//
// Layout: activations are [N][C][X][Y][Z] float32 (Z fastest, the element order of the
// structured mesh), weights [Cout][Cin][3][3][3], zero padding 1, stride 1 or 2.
// Every reduction is a fixed-order two-stage sum, so training is run-to-run reproducible.
//
//   conv forward   y[n,co,o] = b[co] + sum_{ci,t} w[co,ci,t] x[n,ci,s*o + t - 1]   (+ReLU)
//   backward data  dx[n,ci,v] = sum_{co,t : (v - t + 1) = s*o} w[co,ci,t] dy[n,co,o]
//   backward weight dw[co,ci,t] = sum_{n,o} dy[n,co,o] x[n,ci,s*o + t - 1], db = sum dy
// plus ReLU backward, nearest 2x upsampling, channel-range copies (concatenation),
// channel sums and broadcasts (global context), cell-to-node averaging, the mean-squared
// error and the Adam update; and on the solver side the input features, the interpolated
// guess and its energy-optimal scale.
#include <cmath>

#include "common.cuh"

namespace pf {

constexpr int kCOT = 8;  // output channels per thread (forward) / input channels (backward data)

__device__ __forceinline__ long long vidx(int x, int y, int z, int Y, int Z) { return ((long long)x * Y + y) * Z + z; }

// y: one thread = one output voxel x kCOT output channels
__global__ void __launch_bounds__(128) k_conv_fwd(const float* __restrict__ x, int N, int Cin, int X, int Y, int Z,
                                                  const float* __restrict__ w, const float* __restrict__ b, int Cout,
                                                  int s, int relu, float* __restrict__ y, int Xo, int Yo, int Zo) {
    __shared__ float sw[kCOT][27];
    const long long Vo = (long long)Xo * Yo * Zo, Vi = (long long)X * Y * Z;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int co0 = blockIdx.y * kCOT, n = blockIdx.z;
    int ox = 0, oy = 0, oz = 0;
    if (o < Vo) {
        oz = (int)(o % Zo);
        oy = (int)((o / Zo) % Yo);
        ox = (int)(o / ((long long)Yo * Zo));
    }
    float acc[kCOT];
#pragma unroll
    for (int c = 0; c < kCOT; c++) acc[c] = (co0 + c < Cout) ? b[co0 + c] : 0.f;
    for (int ci = 0; ci < Cin; ci++) {
        __syncthreads();
        for (int t = threadIdx.x; t < kCOT * 27; t += blockDim.x) {
            const int c = t / 27, tap = t % 27;
            sw[c][tap] = (co0 + c < Cout) ? w[((long long)(co0 + c) * Cin + ci) * 27 + tap] : 0.f;
        }
        __syncthreads();
        if (o < Vo) {
            const float* xin = x + ((long long)n * Cin + ci) * Vi;
#pragma unroll
            for (int tx = 0; tx < 3; tx++) {
                const int ix = s * ox + tx - 1;
                if (ix < 0 || ix >= X) continue;
#pragma unroll
                for (int ty = 0; ty < 3; ty++) {
                    const int iy = s * oy + ty - 1;
                    if (iy < 0 || iy >= Y) continue;
#pragma unroll
                    for (int tz = 0; tz < 3; tz++) {
                        const int iz = s * oz + tz - 1;
                        if (iz < 0 || iz >= Z) continue;
                        const float xv = __ldg(xin + vidx(ix, iy, iz, Y, Z));
                        const int tap = (tx * 3 + ty) * 3 + tz;
#pragma unroll
                        for (int c = 0; c < kCOT; c++) acc[c] = fmaf(sw[c][tap], xv, acc[c]);
                    }
                }
            }
        }
    }
    if (o < Vo) {
#pragma unroll
        for (int c = 0; c < kCOT; c++)
            if (co0 + c < Cout) {
                float v = acc[c];
                if (relu) v = fmaxf(v, 0.f);
                y[((long long)n * Cout + co0 + c) * Vo + o] = v;
            }
    }
}

// dx: one thread = one input voxel x kCOT input channels
__global__ void __launch_bounds__(128) k_conv_bwd_data(const float* __restrict__ dy, int N, int Cin, int X, int Y, int Z,
                                                       const float* __restrict__ w, int Cout, int s, int accumulate,
                                                       float* __restrict__ dx, int Xo, int Yo, int Zo) {
    __shared__ float sw[kCOT][27];
    const long long Vo = (long long)Xo * Yo * Zo, Vi = (long long)X * Y * Z;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int ci0 = blockIdx.y * kCOT, n = blockIdx.z;
    int vx = 0, vy = 0, vz = 0;
    if (v < Vi) {
        vz = (int)(v % Z);
        vy = (int)((v / Z) % Y);
        vx = (int)(v / ((long long)Y * Z));
    }
    float acc[kCOT];
#pragma unroll
    for (int c = 0; c < kCOT; c++) acc[c] = 0.f;
    for (int co = 0; co < Cout; co++) {
        __syncthreads();
        for (int t = threadIdx.x; t < kCOT * 27; t += blockDim.x) {
            const int c = t / 27, tap = t % 27;
            sw[c][tap] = (ci0 + c < Cin) ? w[((long long)co * Cin + ci0 + c) * 27 + tap] : 0.f;
        }
        __syncthreads();
        if (v < Vi) {
            const float* g = dy + ((long long)n * Cout + co) * Vo;
#pragma unroll
            for (int tx = 0; tx < 3; tx++) {
                const int px = vx - tx + 1;
                if (px < 0 || px % s) continue;
                const int ox = px / s;
                if (ox >= Xo) continue;
#pragma unroll
                for (int ty = 0; ty < 3; ty++) {
                    const int py = vy - ty + 1;
                    if (py < 0 || py % s) continue;
                    const int oy = py / s;
                    if (oy >= Yo) continue;
#pragma unroll
                    for (int tz = 0; tz < 3; tz++) {
                        const int pz = vz - tz + 1;
                        if (pz < 0 || pz % s) continue;
                        const int oz = pz / s;
                        if (oz >= Zo) continue;
                        const float gv = __ldg(g + vidx(ox, oy, oz, Yo, Zo));
                        const int tap = (tx * 3 + ty) * 3 + tz;
#pragma unroll
                        for (int c = 0; c < kCOT; c++) acc[c] = fmaf(sw[c][tap], gv, acc[c]);
                    }
                }
            }
        }
    }
    if (v < Vi) {
#pragma unroll
        for (int c = 0; c < kCOT; c++)
            if (ci0 + c < Cin) {
                float* d = dx + ((long long)n * Cin + ci0 + c) * Vi + v;
                *d = accumulate ? *d + acc[c] : acc[c];
            }
    }
}

// dw partials: block (co, ci, chunk) sums 27 taps over its voxel chunk of all samples
constexpr int kWChunks = 16;
__global__ void __launch_bounds__(256) k_conv_bwd_weight(const float* __restrict__ x, const float* __restrict__ dy, int N,
                                                         int Cin, int X, int Y, int Z, int Cout, int s, int Xo, int Yo,
                                                         int Zo, float* __restrict__ part) {
    __shared__ float red[8][28];
    const int co = blockIdx.x, ci = blockIdx.y, ch = blockIdx.z;
    const long long Vo = (long long)Xo * Yo * Zo, Vi = (long long)X * Y * Z;
    const long long total = (long long)N * Vo;
    const long long per = (total + kWChunks - 1) / kWChunks;
    const long long beg = ch * per, end = beg + per < total ? beg + per : total;
    float acc[28];
#pragma unroll
    for (int t = 0; t < 28; t++) acc[t] = 0.f;
    for (long long q = beg + threadIdx.x; q < end; q += blockDim.x) {
        const int n = (int)(q / Vo);
        const long long o = q - (long long)n * Vo;
        const int oz = (int)(o % Zo), oy = (int)((o / Zo) % Yo), ox = (int)(o / ((long long)Yo * Zo));
        const float g = dy[((long long)n * Cout + co) * Vo + o];
        acc[27] += g;
        const float* xin = x + ((long long)n * Cin + ci) * Vi;
#pragma unroll
        for (int tx = 0; tx < 3; tx++) {
            const int ix = s * ox + tx - 1;
            if (ix < 0 || ix >= X) continue;
#pragma unroll
            for (int ty = 0; ty < 3; ty++) {
                const int iy = s * oy + ty - 1;
                if (iy < 0 || iy >= Y) continue;
#pragma unroll
                for (int tz = 0; tz < 3; tz++) {
                    const int iz = s * oz + tz - 1;
                    if (iz < 0 || iz >= Z) continue;
                    acc[(tx * 3 + ty) * 3 + tz] += g * __ldg(xin + vidx(ix, iy, iz, Y, Z));
                }
            }
        }
    }
    const int wp = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < 28; t++) {
        float v = acc[t];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (l == 0) red[wp][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < 28) {
        float v = 0.f;
        for (int k = 0; k < 8; k++) v += red[k][threadIdx.x];
        part[(((long long)co * Cin + ci) * 28 + threadIdx.x) * kWChunks + ch] = v;
    }
}

// dw[co,ci,t] = sum_chunks part ; db[co] = sum_chunks part[co,0,27]
__global__ void k_conv_bwd_weight_sum(const float* __restrict__ part, int Cin, int Cout, float* __restrict__ dw,
                                      float* __restrict__ db) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nw = (long long)Cout * Cin * 27;
    if (i < nw) {
        const long long co = i / ((long long)Cin * 27), r = i % ((long long)Cin * 27), ci = r / 27, t = r % 27;
        float v = 0.f;
        for (int k = 0; k < kWChunks; k++) v += part[((co * Cin + ci) * 28 + t) * kWChunks + k];
        dw[i] = v;
    } else if (i < nw + Cout && db) {
        const long long co = i - nw;
        float v = 0.f;
        for (int k = 0; k < kWChunks; k++) v += part[((co * Cin + 0) * 28 + 27) * kWChunks + k];
        db[co] = v;
    }
}

__global__ void k_relu_bwd(long long n, const float* __restrict__ y, float* __restrict__ dy) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!(y[i] > 0.f)) dy[i] = 0.f;
}

// nearest 2x upsampling of [N][C][X][Y][Z] into [N][C][2X][2Y][2Z]; backward sums the 8 children
__global__ void k_up2_fwd(long long total, int X, int Y, int Z, const float* __restrict__ x, float* __restrict__ y) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int Z2 = 2 * Z, Y2 = 2 * Y, X2 = 2 * X;
        const long long V2 = (long long)X2 * Y2 * Z2;
        const long long nc = i / V2, v = i % V2;
        const int z = (int)(v % Z2), yy = (int)((v / Z2) % Y2), xx = (int)(v / ((long long)Y2 * Z2));
        y[i] = x[nc * ((long long)X * Y * Z) + vidx(xx / 2, yy / 2, z / 2, Y, Z)];
    }
}
__global__ void k_up2_bwd(long long total, int X, int Y, int Z, const float* __restrict__ dy, float* __restrict__ dx) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long V = (long long)X * Y * Z;
        const long long nc = i / V, v = i % V;
        const int z = (int)(v % Z), yy = (int)((v / Z) % Y), xx = (int)(v / ((long long)Y * Z));
        const int Y2 = 2 * Y, Z2 = 2 * Z;
        const float* g = dy + nc * (8 * V);
        float s = 0.f;
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
                for (int c = 0; c < 2; c++) s += g[vidx(2 * xx + a, 2 * yy + b, 2 * z + c, Y2, Z2)];
        dx[i] = s;
    }
}

// dst[n][c_off + c][v] (+)= src[n][c][v] for c < Csrc (accumulate when acc != 0)
__global__ void k_copy_channels(long long total, int Csrc, long long V, const float* __restrict__ src, int Cdst,
                                int c_off, int acc, float* __restrict__ dst, int reverse) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long n = i / ((long long)Csrc * V), r = i % ((long long)Csrc * V);
        const long long d = (n * Cdst + c_off) * V + r;
        if (!reverse) {
            dst[d] = acc ? dst[d] + src[i] : src[i];
        } else {  // gather back: dst is the small tensor, src the wide one
            dst[i] = acc ? dst[i] + src[d] : src[d];
        }
    }
}

// out[n][c] = scale * sum_v src[n][c_off + c][v]: one block per (n, c), fixed-order sum
__global__ void __launch_bounds__(256) k_channel_sum(int C, long long V, const float* __restrict__ src, int Csrc, int c_off,
                                                     float scale, float* __restrict__ out) {
    __shared__ double red[8];
    const int n = blockIdx.x / C, c = blockIdx.x % C;
    const float* p = src + ((long long)n * Csrc + c_off + c) * V;
    double s = 0.0;
    for (long long v = threadIdx.x; v < V; v += blockDim.x) s += p[v];
    s = block_sum<256>(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = (float)(s * scale);
}
// dst[n][c_off + c][v] (+)= scale * g[n][c]
__global__ void k_channel_bcast(long long total, int C, long long V, const float* __restrict__ g, float scale, int Cdst,
                                int c_off, int acc, float* __restrict__ dst) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long nc = i / V, v = i % V;
        const long long n = nc / C, c = nc % C;
        float* d = dst + (n * Cdst + c_off + c) * V + v;
        const float val = scale * g[nc];
        *d = acc ? *d + val : val;
    }
}

// nodes (X+1)(Y+1)(Z+1) x 3 interleaved by component from cells [N][3][X][Y][Z]: mean of the
// (up to 8) adjacent cells; backward distributes equally
__global__ void k_cell2node_fwd(int N, int X, int Y, int Z, const float* __restrict__ cell, float* __restrict__ node) {
    const long long Nn = (long long)(X + 1) * (Y + 1) * (Z + 1);
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * Nn) return;
    const int n = (int)(i / Nn);
    const long long m = i % Nn;
    // node ordering of the structured mesh: k + nz*(i + nx*j), (x = i, y = j, z = k)
    const int nz = Z + 1, nx = X + 1;
    const int k = (int)(m % nz), ii = (int)((m / nz) % nx), j = (int)(m / ((long long)nz * nx));
    float s[3] = {0.f, 0.f, 0.f};
    int cnt = 0;
    for (int a = -1; a <= 0; a++)
        for (int b = -1; b <= 0; b++)
            for (int c = -1; c <= 0; c++) {
                const int cx = ii + a, cy = j + b, cz = k + c;
                if (cx < 0 || cy < 0 || cz < 0 || cx >= X || cy >= Y || cz >= Z) continue;
                cnt++;
                for (int d = 0; d < 3; d++) s[d] += cell[((long long)n * 3 + d) * ((long long)X * Y * Z) + vidx(cx, cy, cz, Y, Z)];
            }
    for (int d = 0; d < 3; d++) node[((long long)n * Nn + m) * 3 + d] = s[d] / (float)cnt;
}
__global__ void k_cell2node_bwd(int N, int X, int Y, int Z, const float* __restrict__ dnode, float* __restrict__ dcell) {
    const long long V = (long long)X * Y * Z;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * V) return;
    const int n = (int)(i / V);
    const long long v = i % V;
    const int cz = (int)(v % Z), cy = (int)((v / Z) % Y), cx = (int)(v / ((long long)Y * Z));
    const int nz = Z + 1, nx = X + 1;
    const long long Nn = (long long)(X + 1) * (Y + 1) * (Z + 1);
    float s[3] = {0.f, 0.f, 0.f};
    for (int a = 0; a <= 1; a++)
        for (int b = 0; b <= 1; b++)
            for (int c = 0; c <= 1; c++) {
                const int ii = cx + a, j = cy + b, k = cz + c;
                int cnt = 0;
                for (int a2 = -1; a2 <= 0; a2++)
                    for (int b2 = -1; b2 <= 0; b2++)
                        for (int c2 = -1; c2 <= 0; c2++) {
                            const int qx = ii + a2, qy = j + b2, qz = k + c2;
                            if (qx >= 0 && qy >= 0 && qz >= 0 && qx < X && qy < Y && qz < Z) cnt++;
                        }
                const long long m = (long long)k + (long long)nz * (ii + (long long)nx * j);
                for (int d = 0; d < 3; d++) s[d] += dnode[((long long)n * Nn + m) * 3 + d] / (float)cnt;
            }
    for (int d = 0; d < 3; d++) dcell[((long long)n * 3 + d) * V + v] = s[d];
}

// loss = mean((p - t)^2) over n values; grad = 2 (p - t) / n ; partial sums per block
__global__ void __launch_bounds__(256) k_mse(long long n, const float* __restrict__ p, const float* __restrict__ t,
                                             float* __restrict__ g, double* partials) {
    __shared__ double red[8];
    double s = 0.0;
    const float inv = 2.f / (float)n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = p[i] - t[i];
        s += (double)d * d;
        if (g) g[i] = inv * d;
    }
    s = block_sum<256>(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
__global__ void k_mse_final(const double* partials, int np, long long n, double* out) {
    double s = 0.0;
    for (int i = 0; i < np; i++) s += partials[i];
    *out = s / (double)n;
}

__global__ void k_adam(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// ---- the solver side of the network: input features, the guess, its energy-optimal scale ----
//
// A structured mesh of F = (FX, FY, FZ) elements is seen by the network on a cell grid of
// F / P cells (P = 1, 2, 4, ...): cell (cx, cy, cz) covers the fine elements of the block
// [P cx, P cx + P) x ... and the fine nodes of the closed block [P cx, P cx + P] x ....
// Node numbering of the structured mesh: k + nz (i + nx j) for the node at (x, y, z) = (i, j, k).

__device__ __forceinline__ long long node_id(int i, int j, int k, int nx, int nz) {
    return (long long)k + (long long)nz * (i + (long long)nx * j);
}

// max |f| as float bits (non-negative floats order like their bit patterns)
__global__ void k_absmax(long long n, const double* __restrict__ f, unsigned* __restrict__ out) {
    float m = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, (float)fabs(f[i]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));
}

// channels: 0 stiffness E^(1/3) of the block mean, 1-3 the nodal forces of the closed block
// (a node shared with a neighbouring block counts half per shared axis) over max |f|,
// 4 the constrained fraction of the 24 DOFs at the cell's corners, 5-7 the cell-centre
// coordinates scaled to (-1, 1)
__global__ void k_features(int FX, int FY, int FZ, int P, const double* __restrict__ E, const double* __restrict__ f,
                           const uint8_t* __restrict__ node_mask, const unsigned* __restrict__ fmax_bits,
                           float* __restrict__ out) {
    const int X = FX / P, Y = FY / P, Z = FZ / P;
    const long long V = (long long)X * Y * Z;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= V) return;
    const int cz = (int)(c % Z), cy = (int)((c / Z) % Y), cx = (int)(c / ((long long)Y * Z));
    const int nx = FX + 1, nz = FZ + 1;
    double es = 0.0;
    for (int a = 0; a < P; a++)
        for (int b = 0; b < P; b++)
            for (int d = 0; d < P; d++)
                es += E[((long long)(P * cx + a) * FY + (P * cy + b)) * FZ + (P * cz + d)];
    es /= (double)P * P * P;
    double fs[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a <= P; a++) {
        const int i = P * cx + a;
        const double wa = (a == 0 || a == P) && i > 0 && i < FX ? 0.5 : 1.0;
        for (int b = 0; b <= P; b++) {
            const int j = P * cy + b;
            const double wb = wa * ((b == 0 || b == P) && j > 0 && j < FY ? 0.5 : 1.0);
            for (int d = 0; d <= P; d++) {
                const int k = P * cz + d;
                const double w = wb * ((d == 0 || d == P) && k > 0 && k < FZ ? 0.5 : 1.0);
                const long long m = node_id(i, j, k, nx, nz);
                for (int q = 0; q < 3; q++) fs[q] += w * f[3 * m + q];
            }
        }
    }
    const float fm = __uint_as_float(*fmax_bits);
    const float fscale = fm > 0.f ? 1.f / fm : 0.f;
    int ncon = 0;
    if (node_mask)
        for (int a = 0; a <= 1; a++)
            for (int b = 0; b <= 1; b++)
                for (int d = 0; d <= 1; d++)
                    ncon += __popc(node_mask[node_id(P * (cx + a), P * (cy + b), P * (cz + d), nx, nz)] & 7u);
    out[c] = (float)cbrt(es);
    for (int q = 0; q < 3; q++) out[(1 + q) * V + c] = (float)fs[q] * fscale;
    out[4 * V + c] = (float)ncon / 24.f;
    out[5 * V + c] = (2.f * cx + 1.f) / X - 1.f;  // cell-centre coordinates in (-1, 1)
    out[6 * V + c] = (2.f * cy + 1.f) / Y - 1.f;
    out[7 * V + c] = (2.f * cz + 1.f) / Z - 1.f;
}

// fine-node guess: trilinear interpolation of the coarse nodal field (the mesh with F / P
// elements), zero on constrained DOFs
__global__ void k_guess(int FX, int FY, int FZ, int P, const float* __restrict__ cn, const uint8_t* __restrict__ node_mask,
                        double* __restrict__ x0) {
    const int nx = FX + 1, ny = FY + 1, nz = FZ + 1;
    const long long Nf = (long long)nx * ny * nz;
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= Nf) return;
    const int k = (int)(m % nz), i = (int)((m / nz) % nx), j = (int)(m / ((long long)nz * nx));
    const int X = FX / P, Z = FZ / P;
    const int cnx = X + 1, cnz = Z + 1;
    int i0 = i / P, j0 = j / P, k0 = k / P;
    double ti = (double)(i - P * i0) / P, tj = (double)(j - P * j0) / P, tk = (double)(k - P * k0) / P;
    // the last node plane lies on a coarse node: use the cell below it with weight 1
    if (i0 == FX / P) { i0--; ti = 1.0; }
    if (j0 == FY / P) { j0--; tj = 1.0; }
    if (k0 == FZ / P) { k0--; tk = 1.0; }
    double s[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a <= 1; a++)
        for (int b = 0; b <= 1; b++)
            for (int d = 0; d <= 1; d++) {
                const double w = (a ? ti : 1.0 - ti) * (b ? tj : 1.0 - tj) * (d ? tk : 1.0 - tk);
                const long long q = node_id(i0 + a, j0 + b, k0 + d, cnx, cnz);
                for (int e = 0; e < 3; e++) s[e] += w * (double)cn[3 * q + e];
            }
    const unsigned msk = node_mask ? node_mask[m] : 0u;
    for (int e = 0; e < 3; e++) x0[3 * m + e] = (msk >> e) & 1u ? 0.0 : s[e];
}

// x0 *= (x0 . b) / (x0 . K x0): the multiple of x0 with the least energy error; the
// relative residual ||b - alpha K x0|| / ||b|| of the scaled guess follows from the same dots
constexpr int kScaleBlocks = 2 * kNumSM;
__global__ void __launch_bounds__(256) k_scale_partials(long long n, const double* __restrict__ x, const double* __restrict__ kx,
                                                        const double* __restrict__ b, double* __restrict__ part) {
    __shared__ double red[8];
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // x.b, x.Kx, b.b, b.Kx, Kx.Kx
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double xi = x[i], ki = kx[i], bi = b[i];
        s[0] += xi * bi;
        s[1] += xi * ki;
        s[2] += bi * bi;
        s[3] += bi * ki;
        s[4] += ki * ki;
    }
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const double t = block_sum<256>(s[q], red);
        if (threadIdx.x == 0) part[q * kScaleBlocks + blockIdx.x] = t;
    }
}
__global__ void k_scale_apply(long long n, const double* __restrict__ part, double* __restrict__ x,
                              double* __restrict__ out /* alpha, relative residual */) {
    double s[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
        s[q] = 0.0;
        for (int i = 0; i < kScaleBlocks; i++) s[q] += part[q * kScaleBlocks + i];
    }
    const double alpha = s[1] > 0.0 ? s[0] / s[1] : 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const double r2 = fmax(s[2] - 2.0 * alpha * s[3] + alpha * alpha * s[4], 0.0);
        out[0] = alpha;
        out[1] = s[2] > 0.0 ? sqrt(r2 / s[2]) : 0.0;
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] *= alpha;
}

// Energy deficit of the best multiple of y (the Rayleigh-Ritz principle for K u = b):
//   L = 1 - (b.y)^2 / ((y.Ky) c),  c = b.u the compliance of the exact solution,
//   dL/dy = -2 (b.y) / ((y.Ky) c) (b - (b.y) / (y.Ky) Ky)
// which is 1 - cos^2 of the angle between y and u in the energy inner product: the
// energy error left after the guess is scaled by alpha = (y.b) / (y.Ky).
__global__ void __launch_bounds__(256) k_energy_partials(long long n, const double* __restrict__ y,
                                                         const double* __restrict__ ky, const double* __restrict__ b,
                                                         double* __restrict__ part) {
    __shared__ double red[8];
    double sa = 0.0, sq = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        sa += b[i] * y[i];
        sq += y[i] * ky[i];
    }
    sa = block_sum<256>(sa, red);
    sq = block_sum<256>(sq, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sa;
        part[kScaleBlocks + blockIdx.x] = sq;
    }
}
__global__ void k_energy_grad(long long n, const double* __restrict__ part, const double* __restrict__ ky,
                              const double* __restrict__ b, double c, float* __restrict__ grad, double* __restrict__ loss) {
    double a = 0.0, q = 0.0;
    for (int i = 0; i < kScaleBlocks; i++) {
        a += part[i];
        q += part[kScaleBlocks + i];
    }
    const bool ok = q > 0.0 && c > 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *loss = ok ? 1.0 - a * a / (q * c) : 1.0;
    const double s = ok ? -2.0 * a / (q * c) : 0.0, r = ok ? a / q : 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        grad[i] = (float)(s * (b[i] - r * ky[i]));
}

static unsigned gs(long long n) {
    long long b = (n + 255) / 256;
    if (b > 16LL * kNumSM) b = 16LL * kNumSM;
    return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace pf

using namespace pf;

static int out_extent(int n, int s) { return (n - 1) / s + 1; }

extern "C" int pf_cnn_conv3d_fwd_f32(const float* x, int N, int Cin, int X, int Y, int Z, const float* w, const float* b,
                                     int Cout, int stride, int relu, float* y, void* stream) {
    if (!x || !w || !b || !y || N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 || (stride != 1 && stride != 2))
        return fail(PF_BAD_ARG, "pf_cnn_conv3d_fwd_f32: bad argument");
    const int Xo = out_extent(X, stride), Yo = out_extent(Y, stride), Zo = out_extent(Z, stride);
    const long long Vo = (long long)Xo * Yo * Zo;
    dim3 grid((unsigned)((Vo + 127) / 128), (unsigned)((Cout + kCOT - 1) / kCOT), (unsigned)N);
    count_launch();
    k_conv_fwd<<<grid, 128, 0, as_stream(stream)>>>(x, N, Cin, X, Y, Z, w, b, Cout, stride, relu, y, Xo, Yo, Zo);
    PF_LAUNCH_CHECK("conv fwd launch");
    return PF_OK;
}

extern "C" int pf_cnn_conv3d_bwd_data_f32(const float* dy, int N, int Cin, int X, int Y, int Z, const float* w, int Cout,
                                          int stride, int accumulate, float* dx, void* stream) {
    if (!dy || !w || !dx || N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 || (stride != 1 && stride != 2))
        return fail(PF_BAD_ARG, "pf_cnn_conv3d_bwd_data_f32: bad argument");
    const int Xo = out_extent(X, stride), Yo = out_extent(Y, stride), Zo = out_extent(Z, stride);
    const long long Vi = (long long)X * Y * Z;
    dim3 grid((unsigned)((Vi + 127) / 128), (unsigned)((Cin + kCOT - 1) / kCOT), (unsigned)N);
    count_launch();
    k_conv_bwd_data<<<grid, 128, 0, as_stream(stream)>>>(dy, N, Cin, X, Y, Z, w, Cout, stride, accumulate, dx, Xo,
                                                         Yo, Zo);
    PF_LAUNCH_CHECK("conv bwd data launch");
    return PF_OK;
}

extern "C" size_t pf_cnn_conv3d_bwd_weight_workspace(int Cin, int Cout) {
    return (size_t)Cout * Cin * 28 * kWChunks;
}

extern "C" int pf_cnn_conv3d_bwd_weight_f32(const float* x, const float* dy, int N, int Cin, int X, int Y, int Z, int Cout,
                                            int stride, float* dw, float* db, float* work, void* stream) {
    if (!x || !dy || !dw || !work || N < 1 || Cin < 1 || Cout < 1 || X < 1 || Y < 1 || Z < 1 ||
        (stride != 1 && stride != 2))
        return fail(PF_BAD_ARG, "pf_cnn_conv3d_bwd_weight_f32: bad argument");
    const int Xo = out_extent(X, stride), Yo = out_extent(Y, stride), Zo = out_extent(Z, stride);
    cudaStream_t st = as_stream(stream);
    count_launch(2);
    k_conv_bwd_weight<<<dim3(Cout, Cin, kWChunks), 256, 0, st>>>(x, dy, N, Cin, X, Y, Z, Cout, stride, Xo, Yo, Zo, work);
    const long long nt = (long long)Cout * Cin * 27 + Cout;
    k_conv_bwd_weight_sum<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(work, Cin, Cout, dw, db);
    PF_LAUNCH_CHECK("conv bwd weight launch");
    return PF_OK;
}

extern "C" int pf_cnn_relu_bwd_f32(long long n, const float* y, float* dy, void* stream) {
    if (n < 0 || !y || !dy) return fail(PF_BAD_ARG, "pf_cnn_relu_bwd_f32: bad argument");
    count_launch();
    k_relu_bwd<<<gs(n), 256, 0, as_stream(stream)>>>(n, y, dy);
    PF_LAUNCH_CHECK("relu bwd launch");
    return PF_OK;
}

extern "C" int pf_cnn_upsample2_f32(int NC, int X, int Y, int Z, const float* x, float* y, int backward, void* stream) {
    if (NC < 1 || X < 1 || Y < 1 || Z < 1 || !x || !y) return fail(PF_BAD_ARG, "pf_cnn_upsample2_f32: bad argument");
    count_launch();
    if (!backward) {
        const long long total = (long long)NC * 8 * X * Y * Z;
        k_up2_fwd<<<gs(total), 256, 0, as_stream(stream)>>>(total, X, Y, Z, x, y);
    } else {
        const long long total = (long long)NC * X * Y * Z;
        k_up2_bwd<<<gs(total), 256, 0, as_stream(stream)>>>(total, X, Y, Z, x, y);
    }
    PF_LAUNCH_CHECK("upsample launch");
    return PF_OK;
}

extern "C" int pf_cnn_copy_channels_f32(int N, int Csrc, long long V, const float* src, int Cdst, int c_off, int accumulate,
                                        int gather, float* dst, void* stream) {
    if (N < 1 || Csrc < 1 || V < 1 || !src || !dst || c_off < 0 || c_off + Csrc > Cdst)
        return fail(PF_BAD_ARG, "pf_cnn_copy_channels_f32: bad argument");
    const long long total = (long long)N * Csrc * V;
    count_launch();
    k_copy_channels<<<gs(total), 256, 0, as_stream(stream)>>>(total, Csrc, V, src, Cdst, c_off, accumulate, dst, gather);
    PF_LAUNCH_CHECK("copy channels launch");
    return PF_OK;
}

extern "C" int pf_cnn_channel_sum_f32(int N, int C, long long V, const float* src, int Csrc, int c_off, float scale,
                                      float* out, void* stream) {
    if (N < 1 || C < 1 || V < 1 || !src || !out || c_off < 0 || c_off + C > Csrc)
        return fail(PF_BAD_ARG, "pf_cnn_channel_sum_f32: bad argument");
    count_launch();
    k_channel_sum<<<(unsigned)(N * C), 256, 0, as_stream(stream)>>>(C, V, src, Csrc, c_off, scale, out);
    PF_LAUNCH_CHECK("channel sum launch");
    return PF_OK;
}

extern "C" int pf_cnn_channel_bcast_f32(int N, int C, long long V, const float* g, float scale, int Cdst, int c_off,
                                        int accumulate, float* dst, void* stream) {
    if (N < 1 || C < 1 || V < 1 || !g || !dst || c_off < 0 || c_off + C > Cdst)
        return fail(PF_BAD_ARG, "pf_cnn_channel_bcast_f32: bad argument");
    const long long total = (long long)N * C * V;
    count_launch();
    k_channel_bcast<<<gs(total), 256, 0, as_stream(stream)>>>(total, C, V, g, scale, Cdst, c_off, accumulate, dst);
    PF_LAUNCH_CHECK("channel broadcast launch");
    return PF_OK;
}

extern "C" int pf_cnn_cell2node_f32(int N, int X, int Y, int Z, const float* in, float* out, int backward, void* stream) {
    if (N < 1 || X < 1 || Y < 1 || Z < 1 || !in || !out) return fail(PF_BAD_ARG, "pf_cnn_cell2node_f32: bad argument");
    count_launch();
    if (!backward) {
        const long long n = (long long)N * (X + 1) * (Y + 1) * (Z + 1);
        k_cell2node_fwd<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(N, X, Y, Z, in, out);
    } else {
        const long long n = (long long)N * X * Y * Z;
        k_cell2node_bwd<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(N, X, Y, Z, in, out);
    }
    PF_LAUNCH_CHECK("cell2node launch");
    return PF_OK;
}

extern "C" size_t pf_cnn_mse_workspace(long long n) { return (size_t)gs(n < 1 ? 1 : n); }

extern "C" int pf_cnn_mse_f32(long long n, const float* pred, const float* target, float* grad, double* loss,
                              double* work, void* stream) {
    if (n < 1 || !pred || !target || !loss || !work) return fail(PF_BAD_ARG, "pf_cnn_mse_f32: bad argument");
    cudaStream_t st = as_stream(stream);
    const unsigned nb = gs(n);
    count_launch(2);
    k_mse<<<nb, 256, 0, st>>>(n, pred, target, grad, work);
    k_mse_final<<<1, 1, 0, st>>>(work, (int)nb, n, loss);
    PF_LAUNCH_CHECK("mse launch");
    return PF_OK;
}

extern "C" int pf_cnn_adam_f32(long long n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                               float eps, int step, void* stream) {
    if (n < 1 || !p || !g || !m || !v || step < 1) return fail(PF_BAD_ARG, "pf_cnn_adam_f32: bad argument");
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    count_launch();
    k_adam<<<gs(n), 256, 0, as_stream(stream)>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2);
    PF_LAUNCH_CHECK("adam launch");
    return PF_OK;
}

static int fine_grid(const pf_grid* fine, int P, Grid* g, const char* who) {
    int s = validate_grid(fine, g);
    if (s) return s;
    if (g->dim != 3 || P < 1 || g->nel[0] % P || g->nel[1] % P || g->nel[2] % P)
        return fail(PF_BAD_ARG, "%s: 3D grid with every element count divisible by the pooling factor", who);
    return PF_OK;
}

extern "C" int pf_cnn_features_f32(const pf_grid* fine, int P, const double* E, const double* f, const uint8_t* node_mask,
                                   unsigned* work, float* out, void* stream) {
    Grid g;
    int s = fine_grid(fine, P, &g, "pf_cnn_features_f32");
    if (s) return s;
    if (!E || !f || !work || !out) return fail(PF_BAD_ARG, "pf_cnn_features_f32: null pointer");
    cudaStream_t st = as_stream(stream);
    const long long D = 3LL * (g.nel[0] + 1) * (g.nel[1] + 1) * (g.nel[2] + 1);
    const long long V = (long long)(g.nel[0] / P) * (g.nel[1] / P) * (g.nel[2] / P);
    PF_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned), st));
    count_launch(2);
    k_absmax<<<gs(D), 256, 0, st>>>(D, f, work);
    k_features<<<(unsigned)((V + 127) / 128), 128, 0, st>>>(g.nel[0], g.nel[1], g.nel[2], P, E, f, node_mask, work, out);
    PF_LAUNCH_CHECK("features launch");
    return PF_OK;
}

extern "C" int pf_cnn_guess_f64(const pf_grid* fine, int P, const float* coarse_nodes, const uint8_t* node_mask, double* x0,
                                void* stream) {
    Grid g;
    int s = fine_grid(fine, P, &g, "pf_cnn_guess_f64");
    if (s) return s;
    if (!coarse_nodes || !x0) return fail(PF_BAD_ARG, "pf_cnn_guess_f64: null pointer");
    const long long Nf = (long long)(g.nel[0] + 1) * (g.nel[1] + 1) * (g.nel[2] + 1);
    count_launch();
    k_guess<<<(unsigned)((Nf + 255) / 256), 256, 0, as_stream(stream)>>>(g.nel[0], g.nel[1], g.nel[2], P, coarse_nodes,
                                                                          node_mask, x0);
    PF_LAUNCH_CHECK("guess launch");
    return PF_OK;
}

extern "C" size_t pf_cnn_energy_scale_workspace(void) { return 5 * kScaleBlocks + 2; }

extern "C" int pf_cnn_energy_scale_f64(long long n, double* x0, const double* Kx0, const double* b, double* work,
                                       void* stream) {
    if (n < 1 || !x0 || !Kx0 || !b || !work) return fail(PF_BAD_ARG, "pf_cnn_energy_scale_f64: bad argument");
    cudaStream_t st = as_stream(stream);
    count_launch(2);
    k_scale_partials<<<kScaleBlocks, 256, 0, st>>>(n, x0, Kx0, b, work);
    k_scale_apply<<<gs(n), 256, 0, st>>>(n, work, x0, work + 5 * kScaleBlocks);
    PF_LAUNCH_CHECK("energy scale launch");
    return PF_OK;
}

// Choice between two initial guesses a, b of K u = f: each scaled by its energy-optimal
// factor alpha = (x.f) / (x.Kx), the one with the lower energy -(x.f)^2 / (2 x.Kx) (the
// smaller energy-norm error) is written to out (a guess with x.Kx <= 0 counts as the zero
// start).  stats = {alpha, choice (0 = a, 1 = b), energy of a, energy of b}.
__global__ void __launch_bounds__(256) k_select_partials(long long n, const double* __restrict__ xa,
                                                         const double* __restrict__ ka, const double* __restrict__ xb,
                                                         const double* __restrict__ kb, const double* __restrict__ f,
                                                         double* __restrict__ part) {
    __shared__ double red[8];
    double s[4] = {0.0, 0.0, 0.0, 0.0};  // xa.f, xa.Kxa, xb.f, xb.Kxb
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double fi = f[i], a = xa[i], b = xb[i];
        s[0] += a * fi;
        s[1] += a * ka[i];
        s[2] += b * fi;
        s[3] += b * kb[i];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double t = block_sum<256>(s[q], red);
        if (threadIdx.x == 0) part[q * kScaleBlocks + blockIdx.x] = t;
    }
}
__global__ void k_select_apply(long long n, const double* __restrict__ part, const double* xa, const double* xb,
                               double* out, double* __restrict__ stats) {
    double s[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        s[q] = 0.0;
        for (int i = 0; i < kScaleBlocks; i++) s[q] += part[q * kScaleBlocks + i];
    }
    const double ea = s[1] > 0.0 ? -0.5 * s[0] * s[0] / s[1] : 0.0;
    const double eb = s[3] > 0.0 ? -0.5 * s[2] * s[2] / s[3] : 0.0;
    const bool pick_b = eb < ea;
    const double alpha = pick_b ? (s[3] > 0.0 ? s[2] / s[3] : 0.0) : (s[1] > 0.0 ? s[0] / s[1] : 0.0);
    const double* x = pick_b ? xb : xa;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        stats[0] = alpha;
        stats[1] = pick_b ? 1.0 : 0.0;
        stats[2] = ea;
        stats[3] = eb;
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = alpha * x[i];
}

extern "C" size_t pf_cnn_guess_select_workspace(void) { return 4 * kScaleBlocks + 4; }

extern "C" int pf_cnn_guess_select_f64(long long n, const double* xa, const double* Kxa, const double* xb,
                                       const double* Kxb, const double* f, double* out, double* work, void* stream) {
    if (n < 1 || !xa || !Kxa || !xb || !Kxb || !f || !out || !work)
        return fail(PF_BAD_ARG, "pf_cnn_guess_select_f64: bad argument");
    if (out == Kxa || out == Kxb || out == f) return fail(PF_BAD_ARG, "pf_cnn_guess_select_f64: out aliases an input");
    cudaStream_t st = as_stream(stream);
    count_launch(2);
    k_select_partials<<<kScaleBlocks, 256, 0, st>>>(n, xa, Kxa, xb, Kxb, f, work);
    k_select_apply<<<gs(n), 256, 0, st>>>(n, work, xa, xb, out, work + 4 * kScaleBlocks);
    PF_LAUNCH_CHECK("guess select launch");
    return PF_OK;
}

extern "C" size_t pf_cnn_energy_loss_workspace(void) { return 2 * kScaleBlocks; }

extern "C" int pf_cnn_energy_loss_f64(long long n, const double* y, const double* Ky, const double* b, double c,
                                      float* grad, double* loss, double* work, void* stream) {
    if (n < 1 || !y || !Ky || !b || !grad || !loss || !work) return fail(PF_BAD_ARG, "pf_cnn_energy_loss_f64: bad argument");
    cudaStream_t st = as_stream(stream);
    count_launch(2);
    k_energy_partials<<<kScaleBlocks, 256, 0, st>>>(n, y, Ky, b, work);
    k_energy_grad<<<gs(n), 256, 0, st>>>(n, work, Ky, b, c, grad, loss);
    PF_LAUNCH_CHECK("energy loss launch");
    return PF_OK;
}
