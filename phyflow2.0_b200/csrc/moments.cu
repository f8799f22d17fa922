// moments.cu -- FP64 circulation / linear impulse reduction in a fixed order.
//
// Pass 1: MOM_BLOCKS blocks, block b reduces the contiguous range
// [b*chunk, (b+1)*chunk) thread-strided, then a fixed shared-memory tree.
// Pass 2: one block reduces the MOM_BLOCKS partials the same way.  The grid
// does not depend on the device, so the result is bitwise reproducible.
#include "pf_common.cuh"

namespace {

constexpr int MOM_THREADS = 256;
constexpr int MOM_BLOCKS = 592;

struct M4 {
    double s0, sx, sy, sa;
};

__device__ __forceinline__ M4 block_reduce(M4 v, M4 *sm) {
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int s = MOM_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            M4 a = sm[threadIdx.x], b = sm[threadIdx.x + s];
            a.s0 += b.s0;
            a.sx += b.sx;
            a.sy += b.sy;
            a.sa += b.sa;
            sm[threadIdx.x] = a;
        }
        __syncthreads();
    }
    return sm[0];
}

__global__ void __launch_bounds__(MOM_THREADS)
k_moments_partial(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                  const double *__restrict__ g, M4 *__restrict__ part) {
    __shared__ M4 sm[MOM_THREADS];
    const int64_t chunk = (n + MOM_BLOCKS - 1) / MOM_BLOCKS;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = min(n, lo + chunk);
    M4 v = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = lo + threadIdx.x; i < hi; i += MOM_THREADS) {
        const double gi = g[i];
        v.s0 += gi;
        v.sx += gi * x[i];
        v.sy += gi * y[i];
        v.sa += fabs(gi);
    }
    M4 r = block_reduce(v, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void __launch_bounds__(MOM_THREADS)
k_moments_final(const M4 *__restrict__ part, double *__restrict__ out4) {
    __shared__ M4 sm[MOM_THREADS];
    M4 v = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < MOM_BLOCKS; i += MOM_THREADS) {
        v.s0 += part[i].s0;
        v.sx += part[i].sx;
        v.sy += part[i].sy;
        v.sa += part[i].sa;
    }
    M4 r = block_reduce(v, sm);
    if (threadIdx.x == 0) {
        out4[0] = r.s0;
        out4[1] = r.sx;
        out4[2] = r.sy;
        out4[3] = r.sa;
    }
}

}  // namespace

extern "C" pf_status pf_moments(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                const double *g, double *out4, void *stream) {
    PF_RANGE("pf_moments");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_moments: NULL context");
    PF_CHECK_ARG(n >= 0, "pf_moments: negative size");
    PF_CHECK_ARG(out4 != nullptr, "pf_moments: NULL output");
    PF_CHECK_ARG(n == 0 || (x && y && g), "pf_moments: NULL input array");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PF_TRY(pf::arena_reserve(ctx, sizeof(M4) * MOM_BLOCKS + 256));
    M4 *part = static_cast<M4 *>(pf::arena_take(ctx, sizeof(M4) * MOM_BLOCKS));
    k_moments_partial<<<MOM_BLOCKS, MOM_THREADS, 0, st>>>(n, x, y, g, part);
    PF_TRY(pf::launch_status("k_moments_partial"));
    k_moments_final<<<1, MOM_THREADS, 0, st>>>(part, out4);
    return pf::launch_status("k_moments_final");
}
