// Shared definitions for the pyfantom_b200 CUDA library (sm_100a).
//
// Grid conventions follow the reference structured mesh
// (pyFANTOM/core/CUDA/Kernels/_geom.py:23-49):
//   3D node (i,j,k) -> k + nz*(i + nx*j)   (z fastest, then x, then y)
//   3D element      -> (i*nely + j)*nelz + k
//   2D node (i,j)   -> i + nx*j ; 2D element -> i*nely + j
// DOF d of node n lives at n*dof + d.  Dirichlet constraints are carried as one byte per
// node whose bit d marks DOF d (the "node mask").
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/pyfantom_b200.h"

namespace pf {

// ---------------------------------------------------------------------------------------
// error reporting: the last error message is thread-local; entry points return pf_status
// ---------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int fail(int status, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);

#define PF_CUDA(call)                                        \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return pf::check_cuda(_e, #call); \
    } while (0)

#define PF_LAUNCH_CHECK(what)                                 \
    do {                                                      \
        cudaError_t _e = cudaGetLastError();                  \
        if (_e != cudaSuccess) return pf::check_cuda(_e, what); \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Programmatic dependent launch: kernels on the solver's critical path begin with
// pdl_wait() (returns once the previous kernel in the stream has completed and its writes
// are visible; a no-op when the kernel was launched without the attribute) and then
// pdl_trigger() (lets the next kernel be scheduled once every block of this one has
// started), so the launch of kernel k+1 overlaps the tail of kernel k.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// launch a kernel that starts with pdl_wait() with the programmatic-serialisation attribute
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// ---------------------------------------------------------------------------------------
// grid geometry
// ---------------------------------------------------------------------------------------
struct Grid {
    int dim;
    int nel[3];  // elements per axis (x, y, z); nel[2] = 0 in 2D
    int nn[3];   // nodes per axis; nn[2] = 1 in 2D
    long long n_nodes, n_elem;
    int dof;
};

inline Grid make_grid(int dim, const int* nel) {
    Grid g;
    g.dim = dim;
    g.dof = dim;
    g.n_nodes = 1;
    g.n_elem = 1;
    for (int a = 0; a < 3; a++) {
        g.nel[a] = a < dim ? nel[a] : 0;
        g.nn[a] = a < dim ? nel[a] + 1 : 1;
        if (a < dim) {
            g.n_nodes *= g.nn[a];
            g.n_elem *= g.nel[a];
        }
    }
    return g;
}

inline Grid coarse_grid(const Grid& f) {
    int nc[3] = {f.nel[0] / 2, f.nel[1] / 2, f.dim == 3 ? f.nel[2] / 2 : 0};
    return make_grid(f.dim, nc);
}

inline int validate_grid(const pf_grid* g, Grid* out) {
    if (!g) return fail(PF_BAD_ARG, "grid is NULL");
    if (g->dim != 2 && g->dim != 3) return fail(PF_BAD_ARG, "grid dim must be 2 or 3 (got %d)", g->dim);
    for (int a = 0; a < g->dim; a++)
        if (g->nel[a] < 1 || g->nel[a] > (1 << 20))
            return fail(PF_BAD_ARG, "grid nel[%d]=%d out of range", a, g->nel[a]);
    *out = make_grid(g->dim, g->nel);
    if (out->n_nodes * out->dof >= (1LL << 31))
        return fail(PF_BAD_ARG, "grid too large for 32-bit DOF indexing (%lld DOF)", out->n_nodes * out->dof);
    return PF_OK;
}

// ---------------------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block reduction of one double per thread; result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* smem /* >= NT/32 doubles */) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) smem[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NT / 32; i++) s += smem[i];
    }
    __syncthreads();
    return s;
}

// Matvec epilogues.  A matvec kernel produces y = A u at each owned DOF g and then
//   PF_EPI_STORE       out[g] = y
//   PF_EPI_RESID       out[g] = b[g] - y
//   PF_EPI_JACOBI      out[g] = x[g] + w * dinv[g] * (b[g] - y)
//   PF_EPI_JACOBI_ADD  out[g] = xadd[g] + x[g] + w * dinv[g] * (b[g] - y)
// with w = (*omega) * omega_scale.  If dot_partial is set, the block also accumulates
// sum(dot_a[g] * (dot_of_y ? y : out[g])) into dot_partial[block linear index].
enum EpiMode { PF_EPI_STORE = 0, PF_EPI_RESID = 1, PF_EPI_JACOBI = 2, PF_EPI_JACOBI_ADD = 3 };

template <typename T>
struct Epi {
    int mode;
    const T* b;
    const T* x;
    const T* dinv;
    const T* xadd;
    T* out;
    const double* omega;
    double omega_scale;
    double* dot_partial;
    const T* dot_a;
    int dot_of_y;
    const int* skip;  // if non-NULL and *skip != 0 the kernel does nothing (solver finished)
};

template <typename T>
__device__ __forceinline__ T epi_apply(const Epi<T>& e, long long g, T y, T w) {
    switch (e.mode) {
        case PF_EPI_RESID:
            return e.b[g] - y;
        case PF_EPI_JACOBI:
            return e.x[g] + w * e.dinv[g] * (e.b[g] - y);
        case PF_EPI_JACOBI_ADD:
            return e.xadd[g] + e.x[g] + w * e.dinv[g] * (e.b[g] - y);
        default:
            return y;
    }
}

template <typename T>
__device__ __forceinline__ T epi_omega(const Epi<T>& e) {
    if (e.mode == PF_EPI_JACOBI || e.mode == PF_EPI_JACOBI_ADD) return (T)((*e.omega) * e.omega_scale);
    return (T)0;
}

constexpr int kNumSM = 148;

// number of kernels this library has launched since it was loaded (diagnostics)
void count_launch(unsigned long long n = 1);
void uncount_launch(unsigned long long n);
unsigned long long launch_count();

}  // namespace pf
