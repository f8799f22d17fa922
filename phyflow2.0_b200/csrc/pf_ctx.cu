// pf_ctx.cu -- context, scratch arena and error reporting of libpfblob.
#include <mutex>
#include <vector>

#include "pf_common.cuh"

#include <atomic>
#include <cstring>
#include <new>

namespace pf {

static thread_local char g_err[1024] = {0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void clear_error() { g_err[0] = 0; }

static std::atomic<uint64_t> g_launches{0};

void count_launches(uint64_t kernels) { g_launches.fetch_add(kernels, std::memory_order_relaxed); }

cudaError_t graph_kernel_nodes(cudaGraph_t g, int64_t *out) {
    size_t nn = 0;
    cudaError_t e = cudaGraphGetNodes(g, nullptr, &nn);
    if (e != cudaSuccess) return e;
    std::vector<cudaGraphNode_t> nodes(nn);
    e = cudaGraphGetNodes(g, nodes.data(), &nn);
    if (e != cudaSuccess) return e;
    int64_t k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        e = cudaGraphNodeGetType(nd, &t);
        if (e != cudaSuccess) return e;
        if (t == cudaGraphNodeTypeKernel) ++k;
    }
    *out = k;
    return cudaSuccess;
}

pf_status launch_status(const char *what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("launch of %s failed: %s", what, cudaGetErrorString(e));
        return PF_ERR_CUDA;
    }
    return PF_OK;
}

pf_status arena_reserve(pf_ctx *ctx, size_t bytes) {
    ctx->arena.used = 0;
    if (bytes <= ctx->arena.cap) return PF_OK;
    // grow geometrically so that size sweeps do not reallocate every call
    size_t want = ctx->arena.cap ? ctx->arena.cap : (size_t(1) << 20);
    while (want < bytes) want *= 2;
    if (ctx->arena.base) {
        // the old slice may still be read by queued work of an earlier call
        PF_CUDA_TRY(cudaDeviceSynchronize());
        PF_CUDA_TRY(cudaFree(ctx->arena.base));
        ctx->arena.base = nullptr;
        ctx->arena.cap = 0;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        // retry with the exact size before giving up
        e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("scratch arena: cudaMalloc of %zu bytes failed (%s)", bytes,
                      cudaGetErrorString(e));
            return PF_ERR_OOM;
        }
        want = bytes;
    }
    ctx->arena.base = static_cast<char *>(p);
    ctx->arena.cap = want;
    return PF_OK;
}

// Readers of the translation units' bounds words (checked build).  A
// function-local static: units register during library load, in any order.
static std::vector<BoundsReader> &bounds_readers() {
    static std::vector<BoundsReader> v;
    return v;
}
static std::mutex g_bounds_mu;

void bounds_register(BoundsReader r) {
    std::lock_guard<std::mutex> lk(g_bounds_mu);
    bounds_readers().push_back(r);
}

void *arena_take(pf_ctx *ctx, size_t bytes) {
    size_t b = align256(bytes);
    if (ctx->arena.used + b > ctx->arena.cap) return nullptr;
    void *p = ctx->arena.base + ctx->arena.used;
    ctx->arena.used += b;
    return p;
}

}  // namespace pf

extern "C" {

pf_status pf_create(int device, pf_ctx **out) {
    pf::clear_error();
    PF_CHECK_ARG(out != nullptr, "pf_create: out is NULL");
    *out = nullptr;
    int n = 0;
    PF_CUDA_TRY(cudaGetDeviceCount(&n));
    PF_CHECK_ARG(device >= 0 && device < n, "pf_create: device %d out of range (%d devices)",
                 device, n);
    pf::DeviceGuard dg(device);
    pf_ctx *c = new (std::nothrow) pf_ctx();
    if (!c) {
        pf::set_error("pf_create: host allocation failed");
        return PF_ERR_OOM;
    }
    c->device = device;
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        delete c;
        pf::set_error("cudaGetDeviceProperties failed: %s", cudaGetErrorString(e));
        return PF_ERR_CUDA;
    }
    c->num_sms = prop.multiProcessorCount;
    c->smem_optin = prop.sharedMemPerBlockOptin;
    e = cudaMallocHost(&c->host_small, 4096);
    if (e == cudaSuccess) e = cudaMalloc(&c->dev_small, 4096);
    for (int k = 0; k < 8 && e == cudaSuccess; ++k) e = cudaEventCreate(&c->ev[k]);
    if (e != cudaSuccess) {
        if (c->host_small) cudaFreeHost(c->host_small);
        if (c->dev_small) cudaFree(c->dev_small);
        for (int k = 0; k < 8; ++k)
            if (c->ev[k]) cudaEventDestroy(c->ev[k]);
        delete c;
        pf::set_error("context allocation failed: %s", cudaGetErrorString(e));
        return PF_ERR_CUDA;
    }
    cudaMemset(c->dev_small, 0, 4096);
    *out = c;
    return PF_OK;
}

pf_status pf_destroy(pf_ctx *ctx) {
    pf::clear_error();
    if (!ctx) return PF_OK;
    pf::DeviceGuard dg(ctx->device);
    cudaDeviceSynchronize();
    ctx->fmm_plan_hold.reset();
    if (ctx->arena.base) cudaFree(ctx->arena.base);
    if (ctx->host_small) cudaFreeHost(ctx->host_small);
    if (ctx->dev_small) cudaFree(ctx->dev_small);
    if (ctx->rm_rows) cudaFree(ctx->rm_rows);
    for (int k = 0; k < 8; ++k)
        if (ctx->ev[k]) cudaEventDestroy(ctx->ev[k]);
    delete ctx;
    return PF_OK;
}

const char *pf_last_error(void) { return pf::g_err; }

pf_status pf_mem_usage(const pf_ctx *ctx, size_t *bytes) {
    PF_CHECK_ARG(ctx && bytes, "pf_mem_usage: NULL argument");
    *bytes = ctx->arena.cap;
    return PF_OK;
}

pf_status pf_trim(pf_ctx *ctx) {
    PF_CHECK_ARG(ctx, "pf_trim: NULL context");
    pf::DeviceGuard dg(ctx->device);
    if (ctx->arena.base) {
        PF_CUDA_TRY(cudaDeviceSynchronize());
        PF_CUDA_TRY(cudaFree(ctx->arena.base));
    }
    ctx->arena.base = nullptr;
    ctx->arena.cap = 0;
    ctx->arena.used = 0;
    return PF_OK;
}

int pf_version(void) { return PF_VERSION; }

uint64_t pf_kernel_launches(void) { return pf::g_launches.load(std::memory_order_relaxed); }

int pf_bounds_checked(void) {
#ifdef PF_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

pf_status pf_check_bounds(int device) {
    pf::clear_error();
#ifdef PF_BOUNDS_CHECK
    int cur = 0;
    PF_CUDA_TRY(cudaGetDevice(&cur));
    pf::DeviceGuard dg(device >= 0 ? device : cur);
    PF_CUDA_TRY(cudaDeviceSynchronize());
    std::lock_guard<std::mutex> lk(pf::g_bounds_mu);
    for (pf::BoundsReader r : pf::bounds_readers()) {
        pf::BoundsRecord rec;
        if (!r(&rec)) {
            pf::set_error("pf_check_bounds: reading a bounds word failed");
            return PF_ERR_CUDA;
        }
        if (rec.site != 0ull) {
            pf::set_error("bounds check failed at site %llu: index %lld outside [0, %lld)",
                          rec.site, rec.index, rec.limit);
            return PF_ERR_CUDA;
        }
    }
#else
    (void)device;
#endif
    return PF_OK;
}

}  // extern "C"
