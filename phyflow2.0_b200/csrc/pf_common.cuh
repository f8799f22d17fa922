// pf_common.cuh -- shared host/device helpers of libpfblob.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include <cstdarg>
#include <cstdio>
#include <memory>
#include <string>

#include "../../include/pfblob.h"

#define PF_VERSION 10000

namespace pf {

// --------------------------------------------------------------------------
// Error plumbing: every C-ABI entry returns a pf_status and stores a message
// in a thread-local buffer read by pf_last_error().
void set_error(const char *fmt, ...);
void clear_error();

#define PF_CUDA_TRY(expr)                                                         \
    do {                                                                          \
        cudaError_t pf_e_ = (expr);                                               \
        if (pf_e_ != cudaSuccess) {                                               \
            ::pf::set_error("%s failed: %s (%s:%d)", #expr,                       \
                            cudaGetErrorString(pf_e_), __FILE__, __LINE__);       \
            return PF_ERR_CUDA;                                                   \
        }                                                                         \
    } while (0)

#define PF_CHECK_ARG(cond, ...)                                                   \
    do {                                                                          \
        if (!(cond)) {                                                            \
            ::pf::set_error(__VA_ARGS__);                                         \
            return PF_ERR_INVALID_ARG;                                            \
        }                                                                         \
    } while (0)

// --------------------------------------------------------------------------
// NVTX range over one C-ABI call, named after the entry point (ncu --nvtx
// filters on it; with no tool attached NVTX v3 costs one predicted branch).
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};
#define PF_RANGE(name) ::pf::Range pf_range_(name)

// --------------------------------------------------------------------------
// Bounds-checked build (-DPF_BOUNDS_CHECK, libpfblob_checked.so): kernels test
// their data-dependent indices with PF_IDX_OK(i, n, site); a failed test
// records (site, i, n) in a device word of its translation unit -- the first
// one wins -- and the access is skipped, so nothing traps or faults.
// pf_check_bounds() synchronises and reads and clears every unit's word.  In
// the normal build PF_IDX_OK is the constant true and compiles away.
struct BoundsRecord {
    unsigned long long site;  // 0: no failure
    long long index, limit;
};
using BoundsReader = bool (*)(BoundsRecord *rec);  // reads and clears; false on CUDA error
void bounds_register(BoundsReader r);

#define PF_TRY(expr)                                                              \
    do {                                                                          \
        pf_status pf_s_ = (expr);                                                 \
        if (pf_s_ != PF_OK) return pf_s_;                                         \
    } while (0)

// Last launch error of this thread, as a status.  Every kernel launch site
// calls it right after the launch, which also counts the launch.
pf_status launch_status(const char *what);
// Adds kernels launched by other means (a graph launch: its kernel nodes).
void count_launches(uint64_t kernels);
// Kernel nodes of a captured graph.
cudaError_t graph_kernel_nodes(cudaGraph_t g, int64_t *out);

// --------------------------------------------------------------------------
// Device scratch arena: one grow-only allocation per context, carved into
// 256-byte aligned slices per call (stack discipline: reset at call start).
struct Arena {
    char *base = nullptr;
    size_t cap = 0;
    size_t used = 0;
};

}  // namespace pf

struct pf_ctx {
    int device = 0;
    int num_sms = 0;
    size_t smem_optin = 0;
    pf::Arena arena;
    // host-side pinned staging for small device->host reads
    int64_t *host_small = nullptr;
    // the shared FMM plan used by this context's last call (kept alive until
    // the next call replaces it)
    std::shared_ptr<void> fmm_plan_hold;
    // small persistent device buffer (FMM counters) and profiling events
    int64_t *dev_small = nullptr;
    bool fmm_profile = false;
    cudaEvent_t ev[8] = {};
    cudaStream_t last_stream = nullptr;
    pf_fmm_stats last_stats = {};
    // base cells the remesh scratch is sized for (the last window + 25%)
    int64_t rm_cap_base = 0;
    // row / column lists of a compressed remesh window (sparse blob sets)
    void *rm_rows = nullptr;
    size_t rm_rows_cap = 0;
};

namespace pf {

// Bump allocator over a device buffer (scratch of one call or one batch slot).
struct Bump {
    char *base = nullptr;
    size_t cap = 0;
    size_t used = 0;
    void *take(size_t bytes) {
        const size_t b = (bytes + 255) & ~size_t(255);
        if (used + b > cap) return nullptr;
        void *p = base + used;
        used += b;
        return p;
    }
};

// Make sure the arena holds at least `bytes`; may cudaFree/cudaMalloc, which
// synchronises the device.  Done before any kernel of a call is enqueued.
pf_status arena_reserve(pf_ctx *ctx, size_t bytes);
// Carve a slice (after arena_reserve made room).  Returns nullptr if out of room.
void *arena_take(pf_ctx *ctx, size_t bytes);
inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace pf

// --------------------------------------------------------------------------
// Device helpers
namespace pfd {

// Split a double into a float pair (hi + lo == x to ~2^-48 relative).
__device__ __forceinline__ void split_hilo(double x, float &hi, float &lo) {
    hi = __double2float_rn(x);
    lo = __double2float_rn(x - (double)hi);
}

// Knuth TwoSum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// Compensated accumulator: fold a partial sum p into (hi, lo).
__device__ __forceinline__ void comp_add(float &hi, float &lo, float p) {
    float s, e;
    two_sum(hi, p, s, e);
    hi = s;
    lo = __fadd_rn(lo, e);
}

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

}  // namespace pfd

// Per translation unit: the device word of the bounds-checked build and its
// host reader, registered at load time.
#ifdef PF_BOUNDS_CHECK
namespace {
__device__ pf::BoundsRecord pf_bounds_word;

__device__ __noinline__ bool pf_idx_fail(long long i, long long n, int site) {
    if (atomicCAS(&pf_bounds_word.site, 0ull, (unsigned long long)site) == 0ull) {
        pf_bounds_word.index = i;
        pf_bounds_word.limit = n;
    }
    return false;
}

__device__ __forceinline__ bool pf_idx_ok(long long i, long long n, int site) {
    return (i >= 0 && i < n) ? true : pf_idx_fail(i, n, site);
}

bool pf_bounds_read(pf::BoundsRecord *rec) {
    const pf::BoundsRecord zero = {0ull, 0, 0};
    if (cudaMemcpyFromSymbol(rec, pf_bounds_word, sizeof(*rec)) != cudaSuccess) return false;
    if (rec->site != 0ull && cudaMemcpyToSymbol(pf_bounds_word, &zero, sizeof(zero)) != cudaSuccess)
        return false;
    return true;
}

struct PfBoundsRegistration {
    PfBoundsRegistration() { pf::bounds_register(&pf_bounds_read); }
};
PfBoundsRegistration pf_bounds_registration;
}  // namespace
#define PF_IDX_OK(i, n, site) pf_idx_ok((long long)(i), (long long)(n), (site))
#else
#define PF_IDX_OK(i, n, site) true
#endif

