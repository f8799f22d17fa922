// remesh_noalloc.cu -- M4' remesh whose scratch is a fixed buffer owned by the
// library, for callers that cannot allocate device memory.
//
// Who needs it: a process whose device memory is already fully committed to
// another allocator (for example a serving loop that hands all free HBM to its
// own pool and admits work by what is left), or a latency-critical host thread
// that must not trigger the device-wide synchronisation that cudaMalloc and
// cudaFree can cause.  pf_remesh and pf_remesh_window grow a per-context arena
// with cudaMalloc; this entry point instead works inside one static device
// buffer of PF_NOALLOC_SCRATCH_BYTES that every GPU using the library holds
// until the process exits.  It needs no pf_ctx either (creating one allocates).
//
// The same kernels as pf_remesh_window run on that buffer, so results are the
// same as pf_remesh_window's for the same window.
#include <cmath>
#include <mutex>

#include "remesh.cuh"

namespace {

constexpr size_t NOALLOC_BYTES = (size_t)PF_NOALLOC_SCRATCH_BYTES;
constexpr int MAX_DEVICES = 128;

// The scratch.  In host code this name is only a stand-in for the symbol: the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

struct DeviceSetup {
    char *addr = nullptr;  // device address of g_noalloc_scratch in this device's context
    int num_sms = 0;
};

std::mutex g_mu;
DeviceSetup g_setup[MAX_DEVICES];

// Set-up of the current device, once per device (the first call on a device
// does it): the device address of the scratch and the SM count.  With lazy
// module loading (the CUDA default) the first cudaGetSymbolAddress also loads
// the module, which is when the driver commits the buffer's memory.
pf_status device_setup(int device, DeviceSetup *out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (device < 0 || device >= MAX_DEVICES) {
        pf::set_error("pf_remesh_window_noalloc: device %d outside [0, %d)", device, MAX_DEVICES);
        return PF_ERR_INVALID_ARG;
    }
    DeviceSetup &s = g_setup[device];
    if (!s.addr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            pf::set_error("pf_remesh_window_noalloc: cudaGetSymbolAddress failed: %s",
                          cudaGetErrorString(e));
            return PF_ERR_CUDA;
        }
        int sms = 0;
        const cudaError_t e2 = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e2 != cudaSuccess || sms <= 0) {
            pf::set_error("pf_remesh_window_noalloc: SM count query failed: %s",
                          cudaGetErrorString(e2));
            return PF_ERR_CUDA;
        }
        s.num_sms = sms;
        s.addr = static_cast<char *>(p);
    }
    *out = s;
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
    PF_RANGE("pf_remesh_window_noalloc");
    pf::clear_error();
    PF_CHECK_ARG(n >= 0 && n < ((int64_t)1 << 31), "pf_remesh_window_noalloc: bad n");
    PF_CHECK_ARG(h > 0.0 && h < 1e300, "pf_remesh_window_noalloc: h must be positive and finite");
    PF_CHECK_ARG(std::isfinite(xb0) && std::isfinite(yb0) && std::isfinite(c),
                 "pf_remesh_window_noalloc: bounds and c must be finite");
    // each side below 2^30 and the output window below 2^31 cells: the byte
    // counts below cannot overflow
    PF_CHECK_ARG(nbx > 0 && nby > 0 && nbx < ((int64_t)1 << 30) && nby < ((int64_t)1 << 30) &&
                     (nbx + 3) * (nby + 3) < ((int64_t)1 << 31),
                 "pf_remesh_window_noalloc: bad window %lld x %lld", (long long)nbx,
                 (long long)nby);
    PF_CHECK_ARG(ixmin > -((int64_t)1 << 30) && iymin > -((int64_t)1 << 30) &&
                     ixmin + nbx < ((int64_t)1 << 30) && iymin + nby < ((int64_t)1 << 30),
                 "pf_remesh_window_noalloc: window outside +-2^30");
    PF_CHECK_ARG(n == 0 || (x && y && g), "pf_remesh_window_noalloc: NULL input array");
    PF_CHECK_ARG(capacity >= 0 && (capacity == 0 || (x_out && y_out && g_out)),
                 "pf_remesh_window_noalloc: bad output arrays");
    PF_CHECK_ARG(n_out_dev != nullptr, "pf_remesh_window_noalloc: n_out_dev is NULL");
    const pf::RmWindow win{false, (int32_t)ixmin, (int32_t)iymin, nbx, nby, nbx * nby,
                           (nbx + 3) * (nby + 3), 0};
    const size_t need = pf::remesh_scratch_bytes(n, win.cap_base, win.cap_cell, false);
    if (need > NOALLOC_BYTES) {
        pf::set_error("pf_remesh_window_noalloc: %lld blobs on a %lld x %lld window need %zu bytes "
                      "of scratch; the fixed buffer holds %zu (use pf_remesh_window)",
                      (long long)n, (long long)nbx, (long long)nby, need, NOALLOC_BYTES);
        return PF_ERR_INVALID_ARG;
    }
    int device = -1;
    PF_CUDA_TRY(cudaGetDevice(&device));
    DeviceSetup ds;
    PF_TRY(device_setup(device, &ds));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the buffer keeps the previous call's contents: remesh_core zeroes what
    // must start at zero (its head and cell counts) on the stream first
    pf::Bump sc{ds.addr, NOALLOC_BYTES, 0};
    pf::RmHead *hd = nullptr;
    PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, win, capacity, x_out, y_out, g_out,
                           ix_out, iy_out, nullptr, nullptr, st, ds.num_sms, nullptr,
                           pf::REMESH_M4, &hd));
    return pf::remesh_finish(hd, n_out_dev, status_dev, nullptr, nullptr, st);
}
