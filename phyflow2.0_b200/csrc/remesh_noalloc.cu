// remesh_noalloc.cu -- M4' remesh whose scratch is a fixed buffer owned by the
// library, for callers that cannot allocate device memory.
//
// Who needs it: a process whose device memory is already fully committed to
// another allocator (for example a serving loop that hands all free HBM to its
// own pool and admits work by what is left), or a latency-critical host thread
// that must not trigger the device-wide synchronisation that cudaMalloc and
// cudaFree can cause.  pf_remesh and pf_remesh_window grow a per-context arena
// with cudaMalloc; this entry point instead works inside one static device
// buffer of PF_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
// until the process exits.  It needs no pf_ctx either (creating one allocates).
//
// The same kernels as pf_remesh_window run on that buffer, so results are the
// same as pf_remesh_window's for the same window.
#include <cmath>
#include <mutex>

#include "popctl.cuh"

namespace {

constexpr size_t NOALLOC_BYTES = (size_t)PF_NOALLOC_SCRATCH_BYTES;
constexpr size_t NOALLOC_HEAD = 512;  // output count and status words, then the scratch
constexpr int MAX_DEVICES = 128;

// The scratch.  In host code this name is only a stand-in for the symbol: the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

std::mutex g_mu;
void *g_addr[MAX_DEVICES] = {};

__global__ void k_noalloc_finish(const int32_t *__restrict__ total,
                                 const int32_t *__restrict__ bad, int64_t *__restrict__ n_out,
                                 int32_t *__restrict__ status) {
    *n_out = *total;
    if (status) *status = *bad;
}

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does this set-up).
pf_status scratch_address(int device, char **out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (device < 0 || device >= MAX_DEVICES) {
        pf::set_error("pf_remesh_window_noalloc: device %d outside [0, %d)", device, MAX_DEVICES);
        return PF_ERR_INVALID_ARG;
    }
    if (!g_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            pf::set_error("pf_remesh_window_noalloc: cudaGetSymbolAddress failed: %s",
                          cudaGetErrorString(e));
            return PF_ERR_CUDA;
        }
        g_addr[device] = p;
    }
    *out = static_cast<char *>(g_addr[device]);
    return PF_OK;
}

}  // namespace

extern "C" pf_status pf_remesh_window_noalloc(int64_t n, const double *x, const double *y,
                                              const double *g, double h, double xb0, double yb0,
                                              double c, int64_t ixmin, int64_t iymin, int64_t nbx,
                                              int64_t nby, int64_t capacity, double *x_out,
                                              double *y_out, double *g_out, int64_t *ix_out,
                                              int64_t *iy_out, int64_t *n_out_dev,
                                              int32_t *status_dev, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(n >= 0 && n < ((int64_t)1 << 31), "pf_remesh_window_noalloc: bad n");
    PF_CHECK_ARG(h > 0.0 && h < 1e300, "pf_remesh_window_noalloc: h must be positive and finite");
    PF_CHECK_ARG(std::isfinite(xb0) && std::isfinite(yb0) && std::isfinite(c),
                 "pf_remesh_window_noalloc: bounds and c must be finite");
    PF_CHECK_ARG(nbx > 0 && nby > 0 && nbx < ((int64_t)1 << 30) && nby < ((int64_t)1 << 30),
                 "pf_remesh_window_noalloc: bad window %lld x %lld", (long long)nbx,
                 (long long)nby);
    PF_CHECK_ARG(ixmin > -((int64_t)1 << 30) && iymin > -((int64_t)1 << 30) &&
                     ixmin + nbx < ((int64_t)1 << 30) && iymin + nby < ((int64_t)1 << 30),
                 "pf_remesh_window_noalloc: window outside +-2^30");
    PF_CHECK_ARG(n == 0 || (x && y && g), "pf_remesh_window_noalloc: NULL input array");
    PF_CHECK_ARG(capacity >= 0 && (capacity == 0 || (x_out && y_out && g_out)),
                 "pf_remesh_window_noalloc: bad output arrays");
    PF_CHECK_ARG(n_out_dev != nullptr, "pf_remesh_window_noalloc: n_out_dev is NULL");
    const size_t need = NOALLOC_HEAD + pf::remesh_scratch_bytes(n, nbx, nby);
    if (need > NOALLOC_BYTES) {
        pf::set_error("pf_remesh_window_noalloc: %lld blobs on a %lld x %lld window need %zu bytes "
                      "of scratch; the fixed buffer holds %zu (use pf_remesh_window)",
                      (long long)n, (long long)nbx, (long long)nby, need, NOALLOC_BYTES);
        return PF_ERR_INVALID_ARG;
    }
    int device = -1;
    PF_CUDA_TRY(cudaGetDevice(&device));
    char *base = nullptr;
    PF_TRY(scratch_address(device, &base));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int32_t *total = reinterpret_cast<int32_t *>(base);
    int32_t *bad = reinterpret_cast<int32_t *>(base + 256);
    // the buffer keeps the previous call's contents: zero what must start at zero
    PF_CUDA_TRY(cudaMemsetAsync(base, 0, NOALLOC_HEAD, st));
    pf::Bump sc{base + NOALLOC_HEAD, NOALLOC_BYTES - NOALLOC_HEAD, 0};
    if (n > 0)
        PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, (int32_t)ixmin, (int32_t)iymin, nbx,
                               nby, capacity, x_out, y_out, g_out, ix_out, iy_out, total, bad, st));
    k_noalloc_finish<<<1, 1, 0, st>>>(total, bad, n_out_dev, status_dev);
    return pf::launch_status("k_noalloc_finish");
}
