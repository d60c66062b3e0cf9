// Cone density filter on a structured element grid (forward H x and exact adjoint H^T v).
//
// Reference: apply_filter_2D/3D_kernel, get_filter_2D/3D_weights_kernel and
// apply_filter_2D/3D_transpose_kernel (pyFANTOM/core/CUDA/Kernels/filters.cu:1-154):
//   forward  y_e = sum_k w_k x_{e+o_k} / sum_k w_k      (sums over in-bounds taps only)
//   norm_e   = sum over in-bounds taps of w_k
//   adjoint  s_e = sum_k (w_k / norm_{e+o_k}) v_{e+o_k} (the offset set is symmetric)
// Each block stages the tap table (linear offset, per-axis offsets, weight) in shared
// memory; one thread per element, taps in the reference order.
#include "common.cuh"

struct pf_filter {
    pf::Grid grid;
    int n_taps;
    int* d_off;        // n_taps x dim
    double* d_w;       // n_taps
    double* d_norm;    // n_elem normaliser
};

namespace pf {

constexpr int kMaxTaps = 2048;  // keeps the staged tap table under 48 KB of shared memory

template <int DIM, int MODE>  // MODE 0 forward, 1 adjoint, 2 normaliser
__global__ void __launch_bounds__(256) k_filter(int nelx, int nely, int nelz, int K, const int* __restrict__ off,
                                                const double* __restrict__ w, const double* __restrict__ norm,
                                                const double* __restrict__ x, double* __restrict__ y) {
    extern __shared__ unsigned char smem[];
    double* s_w = reinterpret_cast<double*>(smem);
    int* s_o = reinterpret_cast<int*>(s_w + K);
    for (int t = threadIdx.x; t < K; t += blockDim.x) {
        s_w[t] = w[t];
        for (int a = 0; a < DIM; a++) s_o[t * DIM + a] = off[t * DIM + a];
    }
    __syncthreads();
    const long long ne = DIM == 3 ? (long long)nelx * nely * nelz : (long long)nelx * nely;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    int i, j, k = 0;
    const unsigned ue = (unsigned)e;  // element counts stay below 2^31 (validate_grid)
    if (DIM == 3) {
        const unsigned t = ue / (unsigned)nelz;
        k = (int)(ue - t * (unsigned)nelz);
        i = (int)(t / (unsigned)nely);
        j = (int)(t - (unsigned)i * (unsigned)nely);
    } else {
        i = (int)(ue / (unsigned)nely);
        j = (int)(ue - (unsigned)i * (unsigned)nely);
    }
    double sv = 0.0, sw = 0.0;
    for (int t = 0; t < K; t++) {
        const int a = i + s_o[t * DIM], b = j + s_o[t * DIM + 1], c = DIM == 3 ? k + s_o[t * DIM + 2] : 0;
        if (a < 0 || a >= nelx || b < 0 || b >= nely) continue;
        if (DIM == 3 && (c < 0 || c >= nelz)) continue;
        const long long jd = DIM == 3 ? ((long long)a * nely + b) * nelz + c : (long long)a * nely + b;
        if (MODE == 0) {
            sv += s_w[t] * x[jd];
            sw += s_w[t];
        } else if (MODE == 1) {
            sv += (s_w[t] / norm[jd]) * x[jd];
        } else {
            sw += s_w[t];
        }
    }
    if (MODE == 0)
        y[e] = sw > 0 ? sv / sw : 0.0;
    else if (MODE == 1)
        y[e] = sv;
    else
        y[e] = sw;
}

static int launch_filter(const pf_filter* f, int mode, const double* x, double* y, cudaStream_t st) {
    const Grid& g = f->grid;
    const unsigned nb = (unsigned)((g.n_elem + 255) / 256);
    const size_t sm = (size_t)f->n_taps * (sizeof(double) + g.dim * sizeof(int));
    const int nz = g.dim == 3 ? g.nel[2] : 1;
    count_launch();
#define PF_FILTER_CASE(D, M) \
    k_filter<D, M><<<nb, 256, sm, st>>>(g.nel[0], g.nel[1], nz, f->n_taps, f->d_off, f->d_w, f->d_norm, x, y)
    if (g.dim == 3) {
        if (mode == 0) PF_FILTER_CASE(3, 0);
        else if (mode == 1) PF_FILTER_CASE(3, 1);
        else PF_FILTER_CASE(3, 2);
    } else {
        if (mode == 0) PF_FILTER_CASE(2, 0);
        else if (mode == 1) PF_FILTER_CASE(2, 1);
        else PF_FILTER_CASE(2, 2);
    }
#undef PF_FILTER_CASE
    PF_LAUNCH_CHECK("filter launch");
    return PF_OK;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_filter_create(const pf_grid* grid, int n_taps, const int* h_offsets, const double* h_weights,
                                pf_filter** out) {
    if (!out || !h_offsets || !h_weights) return fail(PF_BAD_ARG, "pf_filter_create: NULL argument");
    *out = nullptr;
    Grid g;
    int s = validate_grid(grid, &g);
    if (s) return s;
    if (n_taps < 1 || n_taps > kMaxTaps) return fail(PF_BAD_ARG, "n_taps must be in [1, %d]", kMaxTaps);
    pf_filter* f = new pf_filter();
    f->grid = g;
    f->n_taps = n_taps;
    if (cudaMalloc(&f->d_off, sizeof(int) * n_taps * g.dim) != cudaSuccess ||
        cudaMalloc(&f->d_w, sizeof(double) * n_taps) != cudaSuccess ||
        cudaMalloc(&f->d_norm, sizeof(double) * g.n_elem) != cudaSuccess) {
        cudaGetLastError();
        pf_filter_destroy(f);
        return fail(PF_NO_MEMORY, "filter allocation failed");
    }
    if (cudaMemcpy(f->d_off, h_offsets, sizeof(int) * n_taps * g.dim, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(f->d_w, h_weights, sizeof(double) * n_taps, cudaMemcpyHostToDevice) != cudaSuccess) {
        pf_filter_destroy(f);
        return fail(PF_CUDA_ERROR, "filter upload failed");
    }
    if ((s = launch_filter(f, 2, nullptr, f->d_norm, nullptr)) || (s = check_cuda(cudaDeviceSynchronize(), "filter normaliser"))) {
        pf_filter_destroy(f);
        return s;
    }
    *out = f;
    return PF_OK;
}

extern "C" int pf_filter_destroy(pf_filter* f) {
    if (!f) return PF_OK;
    if (f->d_off) cudaFree(f->d_off);
    if (f->d_w) cudaFree(f->d_w);
    if (f->d_norm) cudaFree(f->d_norm);
    delete f;
    return PF_OK;
}

extern "C" int pf_filter_normalizer_f64(const pf_filter* f, double* out, void* stream) {
    if (!f || !out) return fail(PF_BAD_ARG, "pf_filter_normalizer_f64: NULL argument");
    PF_CUDA(cudaMemcpyAsync(out, f->d_norm, sizeof(double) * f->grid.n_elem, cudaMemcpyDeviceToDevice, as_stream(stream)));
    return PF_OK;
}

extern "C" int pf_filter_fwd_f64(const pf_filter* f, const double* x, double* y, void* stream) {
    if (!f || !x || !y) return fail(PF_BAD_ARG, "pf_filter_fwd_f64: NULL argument");
    return launch_filter(f, 0, x, y, as_stream(stream));
}

extern "C" int pf_filter_adj_f64(const pf_filter* f, const double* x, double* y, void* stream) {
    if (!f || !x || !y) return fail(PF_BAD_ARG, "pf_filter_adj_f64: NULL argument");
    return launch_filter(f, 1, x, y, as_stream(stream));
}
