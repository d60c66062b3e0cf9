#include <cuda_bf16.h>
// C ABI: library info, errors, element operator objects and single-kernel entry points.
#include <atomic>
#include <cstdarg>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "elemop.cuh"
#include "mgkern.cuh"

namespace pf {
long long csr_nnz(const Grid& g);
int launch_construct_csr(const Grid& g, const double* E, const uint8_t* mask, const double* K0_dev, int* row_ptr,
                         int* col, double* val, cudaStream_t st);

static thread_local char g_err[1024] = "";
static std::atomic<unsigned long long> g_launches{0};

void count_launch(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launch(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return PF_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return PF_NO_MEMORY;
    return PF_CUDA_ERROR;
}

// op-owned device buffers for the stand-alone Galerkin entry point
struct OpAux {
    double* K0 = nullptr;
    double* Kc = nullptr;
    uint8_t* elem_flag = nullptr;
    uint8_t* node_flag = nullptr;
};

}  // namespace pf

using namespace pf;

struct pf_op_holder {
    pf_op op;
    OpAux aux;
};

extern "C" int pf_version(void) { return 100; }

extern "C" unsigned long long pf_launch_count(void) { return pf::launch_count(); }

extern "C" const char* pf_last_error(void) { return pf::g_err; }

extern "C" const char* pf_status_string(int s) {
    switch (s) {
        case PF_OK: return "PF_OK";
        case PF_NOT_CONVERGED: return "PF_NOT_CONVERGED";
        case PF_BREAKDOWN: return "PF_BREAKDOWN";
        case PF_NONFINITE: return "PF_NONFINITE";
        case PF_TIMEOUT: return "PF_TIMEOUT";
        case PF_BAD_ARG: return "PF_BAD_ARG";
        case PF_CUDA_ERROR: return "PF_CUDA_ERROR";
        case PF_NO_MEMORY: return "PF_NO_MEMORY";
        case PF_UNSUPPORTED: return "PF_UNSUPPORTED";
        case PF_FACTOR_FAILED: return "PF_FACTOR_FAILED";
        default: return "PF_UNKNOWN";
    }
}

extern "C" int pf_op_create(const pf_grid* grid, const double* h_K0, pf_op** out) {
    if (!out || !h_K0) return fail(PF_BAD_ARG, "pf_op_create: NULL argument");
    *out = nullptr;
    Grid g;
    int s = validate_grid(grid, &g);
    if (s) return s;
    const int nd = (g.dim == 3 ? 8 : 4) * g.dim;
    for (int i = 0; i < nd * nd; i++)
        if (!std::isfinite(h_K0[i])) return fail(PF_NONFINITE, "K0 has a non-finite entry at %d", i);
    double kmax = 0.0;
    for (int i = 0; i < nd * nd; i++) kmax = fmax(kmax, fabs(h_K0[i]));
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < i; j++)
            if (fabs(h_K0[i * nd + j] - h_K0[j * nd + i]) > 1e-12 * kmax)
                return fail(PF_BAD_ARG, "K0 is not symmetric (entry %d,%d)", i, j);
    auto* h = new pf_op_holder();
    pf_op* op = &h->op;
    op->grid = g;
    memset(op->K0, 0, sizeof(op->K0));
    memcpy(op->K0, h_K0, sizeof(double) * nd * nd);
    op->variant = 0;
    if ((s = op_factorise(op))) {
        delete h;
        return s;
    }
    // device copies for the stand-alone Galerkin entry point
    const int nc = g.dim == 3 ? 8 : 4;
    std::vector<double> Kc((size_t)nc * nd * nd);
    galerkin_child_matrices(g.dim, op->K0, Kc.data());
    const Grid g1 = coarse_grid(g);
    if (cudaMalloc(&h->aux.K0, sizeof(double) * nd * nd) != cudaSuccess ||
        cudaMalloc(&h->aux.Kc, sizeof(double) * Kc.size()) != cudaSuccess ||
        cudaMalloc(&h->aux.elem_flag, (size_t)(g1.n_elem > 0 ? g1.n_elem : 1)) != cudaSuccess ||
        cudaMalloc(&h->aux.node_flag, (size_t)g1.n_nodes) != cudaSuccess) {
        cudaGetLastError();
        pf_op_destroy(op);
        return fail(PF_NO_MEMORY, "pf_op_create: allocation failed");
    }
    if (cudaMemcpy(h->aux.K0, op->K0, sizeof(double) * nd * nd, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->aux.Kc, Kc.data(), sizeof(double) * Kc.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        pf_op_destroy(op);
        return fail(PF_CUDA_ERROR, "pf_op_create: upload failed");
    }
    *out = op;
    return PF_OK;
}

static pf_op_holder* holder(const pf_op* op) {
    return reinterpret_cast<pf_op_holder*>(const_cast<pf_op*>(op));
}

extern "C" int pf_op_destroy(pf_op* op) {
    if (!op) return PF_OK;
    pf_op_holder* h = holder(op);
    for (void* p : {(void*)h->aux.K0, (void*)h->aux.Kc, (void*)h->aux.elem_flag, (void*)h->aux.node_flag})
        if (p) cudaFree(p);
    delete h;
    return PF_OK;
}

extern "C" long long pf_csr_nnz(const pf_op* op) { return op ? pf::csr_nnz(op->grid) : -1; }

extern "C" int pf_construct_csr_f64(const pf_op* op, const double* E, const uint8_t* node_mask, int* row_ptr, int* col,
                                    double* val, void* stream) {
    if (!op || !E || !row_ptr || !col || !val) return fail(PF_BAD_ARG, "pf_construct_csr_f64: NULL argument");
    return launch_construct_csr(op->grid, E, node_mask, holder(op)->aux.K0, row_ptr, col, val, as_stream(stream));
}

extern "C" int pf_pack_mask(const pf_op* op, const uint8_t* con_dof, uint8_t* node_mask, void* stream) {
    if (!op || !con_dof || !node_mask) return fail(PF_BAD_ARG, "pf_pack_mask: NULL argument");
    return launch_pack_mask(op, con_dof, node_mask, as_stream(stream));
}

static Epi<double> store_epi(double* y) {
    Epi<double> e;
    memset(&e, 0, sizeof(e));
    e.mode = PF_EPI_STORE;
    e.out = y;
    e.omega_scale = 1.0;
    return e;
}

extern "C" int pf_matvec_f64(const pf_op* op, const double* E, const double* u, const uint8_t* node_mask, double* y,
                             void* stream) {
    if (!op || !E || !u || !y) return fail(PF_BAD_ARG, "pf_matvec_f64: NULL argument");
    if (u == y) return fail(PF_BAD_ARG, "pf_matvec_f64: u and y must not alias");
    return launch_fine_matvec<double, double>(op, E, u, node_mask, store_epi(y), as_stream(stream));
}

extern "C" int pf_matvec_f32(const pf_op* op, const float* E, const float* u, const uint8_t* node_mask, float* y,
                             void* stream) {
    if (!op || !E || !u || !y) return fail(PF_BAD_ARG, "pf_matvec_f32: NULL argument");
    if (u == y) return fail(PF_BAD_ARG, "pf_matvec_f32: u and y must not alias");
    Epi<float> e;
    memset(&e, 0, sizeof(e));
    e.mode = PF_EPI_STORE;
    e.out = y;
    e.omega_scale = 1.0;
    return launch_fine_matvec<float, float>(op, E, u, node_mask, e, as_stream(stream));
}

extern "C" int pf_op_set_variant(pf_op* op, int variant) {
    if (!op || variant < 0 || variant > 1) return fail(PF_BAD_ARG, "pf_op_set_variant: variant must be 0 or 1");
    op->variant = variant;
    return PF_OK;
}

extern "C" int pf_matvec_f32_bf16(const pf_op* op, const uint16_t* E_bf16, const float* u, const uint8_t* node_mask,
                                  float* y, void* stream) {
    if (!op || !E_bf16 || !u || !y) return fail(PF_BAD_ARG, "pf_matvec_f32_bf16: NULL argument");
    if (u == y) return fail(PF_BAD_ARG, "pf_matvec_f32_bf16: u and y must not alias");
    Epi<float> e;
    memset(&e, 0, sizeof(e));
    e.mode = PF_EPI_STORE;
    e.out = y;
    e.omega_scale = 1.0;
    return launch_fine_matvec<float, __nv_bfloat16>(op, reinterpret_cast<const __nv_bfloat16*>(E_bf16), u, node_mask,
                                                    e, as_stream(stream));
}

extern "C" int pf_diagonal_f64(const pf_op* op, const double* E, const uint8_t* node_mask, double* d, void* stream) {
    if (!op || !E || !d) return fail(PF_BAD_ARG, "pf_diagonal_f64: NULL argument");
    return launch_diagonal<double>(op, E, node_mask, d, as_stream(stream));
}

extern "C" int pf_sensitivity_f64(const pf_op* op, const double* U, double* dk, void* stream) {
    if (!op || !U || !dk) return fail(PF_BAD_ARG, "pf_sensitivity_f64: NULL argument");
    return launch_sensitivity(op, U, dk, as_stream(stream));
}

extern "C" int pf_adjoint_f64(const pf_op* op, const double* U, const double* rho, const pf_simp_params* p,
                              double scale, double* out, void* stream) {
    if (!op || !U || !rho || !p || !out) return fail(PF_BAD_ARG, "pf_adjoint_f64: NULL argument");
    return launch_adjoint(op, U, rho, *p, scale, out, as_stream(stream));
}

// a fine grid with a coarse level: at least two elements per axis (the coarse grid floors
// nel / 2, core/CUDA/_mgm.py:24-27)
static int coarsenable_grid(const pf_grid* fine, Grid* g) {
    int s = validate_grid(fine, g);
    if (s) return s;
    for (int a = 0; a < g->dim; a++)
        if (g->nel[a] < 2) return fail(PF_BAD_ARG, "fine grid nel[%d]=%d has no coarse level", a, g->nel[a]);
    return PF_OK;
}

extern "C" int pf_restrict_f64(const pf_grid* fine, const double* vf, double* vc, void* stream) {
    Grid g;
    int s = coarsenable_grid(fine, &g);
    if (s) return s;
    if (!vf || !vc) return fail(PF_BAD_ARG, "pf_restrict_f64: NULL argument");
    return launch_restrict<double, double>(g, vf, vc, nullptr, as_stream(stream));
}

extern "C" int pf_prolong_f64(const pf_grid* fine, const double* vc, double* vf, void* stream) {
    Grid g;
    int s = coarsenable_grid(fine, &g);
    if (s) return s;
    if (!vf || !vc) return fail(PF_BAD_ARG, "pf_prolong_f64: NULL argument");
    return launch_prolong<double>(g, vc, vf, nullptr, as_stream(stream));
}

extern "C" size_t pf_stencil_size(const pf_grid* grid) {
    Grid g;
    if (validate_grid(grid, &g)) return 0;
    return (size_t)g.n_nodes * (g.dim == 3 ? 27 : 9) * g.dim * g.dim;
}

extern "C" int pf_galerkin_l0_f64(const pf_op* op, const double* E, const uint8_t* node_mask, double* A_coarse,
                                  void* stream) {
    if (!op || !E || !A_coarse) return fail(PF_BAD_ARG, "pf_galerkin_l0_f64: NULL argument");
    const Grid& g = op->grid;
    for (int a = 0; a < g.dim; a++)
        if (g.nel[a] < 2) return fail(PF_BAD_ARG, "fine grid nel[%d]=%d has no coarse level", a, g.nel[a]);
    pf_op_holder* h = holder(op);
    cudaStream_t st = as_stream(stream);
    const Grid g1 = coarse_grid(g);
    int s;
    if (node_mask) {
        if ((s = launch_coarse_flags(g, node_mask, h->aux.elem_flag, h->aux.node_flag, st))) return s;
    } else {
        PF_CUDA(cudaMemsetAsync(h->aux.elem_flag, 0, (size_t)g1.n_elem, st));
        PF_CUDA(cudaMemsetAsync(h->aux.node_flag, 0, (size_t)g1.n_nodes, st));
    }
    return launch_galerkin_l0(g, E, node_mask, h->aux.elem_flag, h->aux.node_flag, h->aux.K0, h->aux.Kc, A_coarse, st);
}

extern "C" int pf_galerkin_l1p_f64(const pf_grid* fine, const double* A_fine, double* A_coarse, void* stream) {
    Grid g;
    int s = coarsenable_grid(fine, &g);
    if (s) return s;
    if (!A_fine || !A_coarse) return fail(PF_BAD_ARG, "pf_galerkin_l1p_f64: NULL argument");
    return launch_galerkin_l1p(g, A_fine, A_coarse, as_stream(stream));
}

extern "C" int pf_stencil_matvec_f64(const pf_grid* grid, const double* A, const double* u, double* y, void* stream) {
    Grid g;
    int s = validate_grid(grid, &g);
    if (s) return s;
    if (!A || !u || !y) return fail(PF_BAD_ARG, "pf_stencil_matvec_f64: NULL argument");
    if (u == y) return fail(PF_BAD_ARG, "pf_stencil_matvec_f64: u and y must not alias");
    return launch_stencil_matvec<double>(g, A, u, store_epi(y), as_stream(stream));
}
