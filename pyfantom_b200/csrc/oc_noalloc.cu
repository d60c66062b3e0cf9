// OC update that allocates nothing: the scratch lives in a static device array.
//
// Who needs this: callers that cannot call cudaMalloc on the path where they run the OC
// step - plugins hosted by a framework that owns the device memory (its caching allocator
// may hold nearly all of it, and the plugin must not allocate behind its back), and
// per-iteration callbacks with a latency budget, where a device allocation (which
// synchronises the device) is not acceptable.  The regular pf_oc_update_f64 asks such
// callers for a workspace they cannot provide.
//
// The scratch is a file-scope __device__ array sized for PF_OC_NOALLOC_MAX_ELEMS
// elements (16.9 MB); every GPU that loads this library holds it until the process exits.
// Host code cannot use the array's name as a device address, so the first call on each
// device resolves it with cudaGetSymbolAddress while that device is current and keeps
// the pointer; that first call may also load the library's device code.  A
// cudaDeviceReset invalidates the kept pointer: the entry point must not be called again
// in that process.  All calls share the array and it keeps the contents of the last
// call; the kernels initialise every value they read
// (the bisection state and all partial sums are written before use), so nothing needs
// clearing between calls.  With a non-NULL h_out the call copies the result scalars to
// the host and waits for the stream.  Calls that overlap on the GPU (different streams
// without ordering) race on the array.
#include <mutex>

#include "common.cuh"

namespace pf {
size_t oc_workspace(long long n);
int oc_update(long long n, const double* x, const double* df, const double* dg, double vf, double move,
              double* x_new, double* work, double* h_out, cudaStream_t st);
}  // namespace pf

namespace {

// ocP for up to PF_OC_NOALLOC_MAX_ELEMS elements + per-block partial sums + bisection state
constexpr size_t kScratchDoubles = (size_t)PF_OC_NOALLOC_MAX_ELEMS + 16384;
__device__ __align__(256) double g_oc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// device address of the scratch for the current device (resolved once per device)
int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return pf::check_cuda(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return pf::fail(PF_UNSUPPORTED, "device ordinal %d >= %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_oc_scratch);
        if (e != cudaSuccess) return pf::check_cuda(e, "cudaGetSymbolAddress(OC scratch)");
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return PF_OK;
}

}  // namespace

extern "C" int pf_oc_update_noalloc_f64(long long n, const double* x, const double* df, const double* dg, double vf,
                                        double move, double* x_new, double* h_out, void* stream) {
    if (n < 1 || !x || !df || !dg || !x_new) return pf::fail(PF_BAD_ARG, "pf_oc_update_noalloc_f64: bad argument");
    if (n > PF_OC_NOALLOC_MAX_ELEMS)
        return pf::fail(PF_BAD_ARG,
                        "pf_oc_update_noalloc_f64: %lld elements exceed the static scratch limit of %d; use "
                        "pf_oc_update_f64 with a workspace of pf_oc_workspace_size(n) doubles",
                        n, PF_OC_NOALLOC_MAX_ELEMS);
    if (!(move >= 0.0)) return pf::fail(PF_BAD_ARG, "move must be >= 0");
    if (pf::oc_workspace(n) > kScratchDoubles)
        return pf::fail(PF_BAD_ARG, "pf_oc_update_noalloc_f64: scratch layout exceeds the static array");
    double* scratch = nullptr;
    int s = scratch_for_current_device(&scratch);
    if (s) return s;
    return pf::oc_update(n, x, df, dg, vf, move, x_new, scratch, h_out, pf::as_stream(stream));
}
