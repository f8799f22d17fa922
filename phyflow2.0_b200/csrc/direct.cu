// direct.cu -- Gaussian-blob Biot-Savart velocity by direct summation.
//
// One simulation per launch (the plain path).  Each CTA owns DT_THREADS*TPT
// targets (TPT per thread, coalesced) and streams a range of sources through
// shared memory in tiles of DT_THREADS blobs, converted on load from FP64 to
// hi/lo float pairs.  Per thread the pair sums run in FP32 over chunks of 32
// sources and are folded into a TwoSum-compensated (hi, lo) accumulator
// after each chunk.
//
// Source splits: unless the target tiles alone fill the device several times
// over, the sources are cut into S contiguous segments (direct_split, a
// function of the two sizes and the device's resident CTA count), CTA (tile, s) writes its (hi, lo) pairs to a partial buffer, and
// k_direct_reduce adds the S partials of each target in segment order in
// FP64.  The batched kernel uses the same segments, so a blob set gets
// bitwise the same velocities alone and in a batch.
//
// Replaces vv2par_kernel (src/cpp/blobs/cuda/vv2parGauss_gpu/
// vv2parGauss_device.cu:107-162: FP64, one target per thread, 2 exp per pair,
// targets padded to a multiple of the block size by the Python caller).  The
// CUTOFF variant sums the cutoff kernel g / (r^2 + sigma^2) of vv2par_C_cpu
// (src/cpp/blobs/c/vv2par_C/vv2par_C_cpu.c:135-151) and its GPU twin
// (src/cpp/blobs/cuda/vv2par_gpu/vv2par_device.cu:59-70) the same way.
#include "direct_api.cuh"
#include "gauss_pair.cuh"

#include <algorithm>
#include <atomic>
#include <climits>

namespace {

constexpr int DT_THREADS = 256;
constexpr int DT_CHUNK = 32;
constexpr double INV_2PI = 0.15915494309189535;  // 0.5/pi
constexpr int64_t DT_TILE = DT_THREADS * 2;      // targets per CTA

// One CTA computes the 2*DT_THREADS targets of tile `tile`: each thread owns
// targets base and base + DT_THREADS and evaluates both against every source
// with the packed f32x2 pair arithmetic (gauss_pair.cuh); CUTOFF: the cutoff
// kernel with core size squared s2.
// Sources [s_begin, s_end) only; with `part` non-null the (hi, lo) sums go to
// part[split * nt + target] instead of the velocities.
template <bool CUTOFF = false>
__device__ __forceinline__ void direct_tile(const double *__restrict__ xs,
                                            const double *__restrict__ ys,
                                            const double *__restrict__ gs, int64_t s_begin,
                                            int64_t s_end, const double *__restrict__ xt,
                                            const double *__restrict__ yt, int64_t nt,
                                            const pfd::GaussParams &gp, double *__restrict__ vx,
                                            double *__restrict__ vy, float4 *__restrict__ part,
                                            int64_t split, int64_t tile, ulonglong2 *s_hi,
                                            ulonglong2 *s_lo, unsigned long long *s_g2,
                                            float s2 = 0.f) {
    const int64_t base = tile * DT_TILE + threadIdx.x;
    float th[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int64_t i = base + (int64_t)j * DT_THREADS;
        double x = 0.0, y = 0.0;
        if (i < nt) {
            x = xt[i];
            y = yt[i];
        }
        pfd::split_hilo(x, th[j][0], th[j][2]);
        pfd::split_hilo(y, th[j][1], th[j][3]);
    }
    const pfd::f32x2 txh = pfd::pack2(th[0][0], th[1][0]), tyh = pfd::pack2(th[0][1], th[1][1]);
    const pfd::f32x2 txl = pfd::pack2(th[0][2], th[1][2]), tyl = pfd::pack2(th[0][3], th[1][3]);
    const pfd::GaussParams2 gp2 = pfd::make_params2(gp);
    const pfd::f32x2 s22 = pfd::pack2(s2, s2);
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};

    for (int64_t t0 = s_begin; t0 < s_end; t0 += DT_THREADS) {
        const int64_t s = t0 + threadIdx.x;
        double x = 0.0, y = 0.0, g = 0.0;  // padding blobs carry g = 0
        if (s < s_end) {
            x = xs[s];
            y = ys[s];
            g = gs[s];
        }
        float xh, xl, yh, yl;
        pfd::split_hilo(x, xh, xl);
        pfd::split_hilo(y, yh, yl);
        const float gf = (float)g;
        __syncthreads();
        s_hi[threadIdx.x] = make_ulonglong2(pfd::pack2(xh, xh), pfd::pack2(yh, yh));
        s_lo[threadIdx.x] = make_ulonglong2(pfd::pack2(xl, xl), pfd::pack2(yl, yl));
        s_g2[threadIdx.x] = pfd::pack2(gf, gf);
        __syncthreads();
        const int nvalid = (int)min((int64_t)DT_THREADS, s_end - t0);
        for (int c0 = 0; c0 < nvalid; c0 += DT_CHUNK) {
            pfd::f32x2 nx = 0ull, ny = 0ull;
#pragma unroll 4
            for (int k = 0; k < DT_CHUNK; ++k) {
                if (CUTOFF)
                    pfd::pair2_cutoff(s_hi[c0 + k], s_lo[c0 + k], s_g2[c0 + k], txh, tyh, txl, tyl,
                                      s22, nx, ny);
                else
                    pfd::pair2(s_hi[c0 + k], s_lo[c0 + k], s_g2[c0 + k], txh, tyh, txl, tyl, gp2,
                               nx, ny);
            }
            float nxa, nxb, nya, nyb;
            pfd::unpack2(nx, nxa, nxb);
            pfd::unpack2(ny, nya, nyb);
            pfd::comp_add(acc[0], acc[1], -nxa);
            pfd::comp_add(acc[2], acc[3], nya);
            pfd::comp_add(acc[4], acc[5], -nxb);
            pfd::comp_add(acc[6], acc[7], nyb);
        }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int64_t i = base + (int64_t)j * DT_THREADS;
        if (i >= nt) continue;
        if (part) {
            part[split * nt + i] = make_float4(acc[4 * j], acc[4 * j + 1], acc[4 * j + 2],
                                               acc[4 * j + 3]);
        } else {
            vx[i] = INV_2PI * ((double)acc[4 * j] + (double)acc[4 * j + 1]);
            vy[i] = INV_2PI * ((double)acc[4 * j + 2] + (double)acc[4 * j + 3]);
        }
    }
}

// v = 1/(2 pi) * sum over segments s = 0..S-1 of (hi_s + lo_s), in FP64.
__device__ __forceinline__ void reduce_target(const float4 *__restrict__ part, int64_t nt,
                                              int splits, int64_t i, double *__restrict__ vx,
                                              double *__restrict__ vy) {
    double sx = 0.0, sy = 0.0;
    for (int s = 0; s < splits; ++s) {
        const float4 p = part[(int64_t)s * nt + i];
        sx += (double)p.x + (double)p.y;
        sy += (double)p.z + (double)p.w;
    }
    vx[i] = INV_2PI * sx;
    vy[i] = INV_2PI * sy;
}

__global__ void __launch_bounds__(DT_THREADS)
k_direct_reduce(const float4 *__restrict__ part, int64_t nt, int splits, double *__restrict__ vx,
                double *__restrict__ vy) {
    const int64_t i = (int64_t)blockIdx.x * DT_THREADS + threadIdx.x;
    if (i < nt) reduce_target(part, nt, splits, i, vx, vy);
}

// grid (target tiles, source segments); one segment = the plain sum.
template <int TPT, bool CUTOFF = false>
__global__ void __launch_bounds__(DT_THREADS)
k_direct_gauss(const double *__restrict__ xs, const double *__restrict__ ys,
               const double *__restrict__ gs, int64_t ns, int64_t seg,
               const double *__restrict__ xt, const double *__restrict__ yt, int64_t nt,
               pfd::GaussParams gp, double *__restrict__ vx, double *__restrict__ vy,
               float4 *__restrict__ part, float s2 = 0.f) {
    static_assert(TPT == 2, "two targets per thread (packed pairs)");
    __shared__ ulonglong2 s_hi[DT_THREADS];  // {x_hi, x_hi}, {y_hi, y_hi}
    __shared__ ulonglong2 s_lo[DT_THREADS];  // {x_lo, x_lo}, {y_lo, y_lo}
    __shared__ unsigned long long s_g2[DT_THREADS];
    const int64_t s0 = (int64_t)blockIdx.y * seg;
    direct_tile<CUTOFF>(xs, ys, gs, s0, min(ns, s0 + seg), xt, yt, nt, gp, vx, vy, part,
                        blockIdx.y, blockIdx.x, s_hi, s_lo, s_g2, s2);
}

// Persistent batched direct sum: CTAs take (instance, target tile) items from
// a device counter until the list is exhausted.  Items are ordered by cost,
// largest first; each item is computed by one CTA, so results do not depend
// on which CTA takes it.
__global__ void __launch_bounds__(DT_THREADS, 4)
k_direct_batch(const pf::DirectInstance *__restrict__ inst, const int2 *__restrict__ items,
               int n_items, int *__restrict__ counter) {
    __shared__ ulonglong2 s_hi[DT_THREADS];
    __shared__ ulonglong2 s_lo[DT_THREADS];
    __shared__ unsigned long long s_g2[DT_THREADS];
    __shared__ int s_item;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const int2 w = items[it];
        const pf::DirectInstance d = inst[w.x];
        const int64_t tile = w.y / d.splits, sp = w.y - tile * d.splits;
        const int64_t s0 = sp * d.seg;
        direct_tile(d.x, d.y, d.g, s0, min(d.n, s0 + d.seg), d.xt, d.yt, d.nt, d.gp, d.vx, d.vy,
                    d.splits > 1 ? d.part : nullptr, sp, tile, s_hi, s_lo, s_g2);
    }
}

// Batched reduction of split instances: one CTA per (instance, target tile).
__global__ void __launch_bounds__(DT_THREADS)
k_direct_reduce_batch(const pf::DirectInstance *__restrict__ inst,
                      const int2 *__restrict__ items) {
    const int2 w = items[blockIdx.x];
    const pf::DirectInstance d = inst[w.x];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int64_t i = (int64_t)w.y * DT_TILE + j * DT_THREADS + threadIdx.x;
        if (i < d.nt) reduce_target(d.part, d.nt, d.splits, i, d.vx, d.vy);
    }
}

}  // namespace

namespace pf {

// k_direct_gauss CTAs resident on the whole current device (cached per
// device; host threads may race to fill an entry, all with the same value).
static int64_t direct_resident_ctas() {
    static std::atomic<int64_t> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DT_SPLIT_CTAS;
    int64_t v = cached[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        int per_sm = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_direct_gauss<2, false>,
                                                          DT_THREADS, 0) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            per_sm <= 0 || sms <= 0) {
            cudaGetLastError();
            return DT_SPLIT_CTAS;
        }
        v = (int64_t)per_sm * sms;
        cached[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// Segments of at least DT_SPLIT_MIN_SRC sources (at most DT_SPLIT_MAX of
// them), in whole 32-source chunks, chosen to minimise the launch's critical
// path: the full waves of resident CTAs times the sources each CTA runs.  A
// grid just above one wave would leave its last CTAs running alone.
DirectSplit direct_split(int64_t ns, int64_t nt) {
    const int64_t tiles = ceil_div(nt, DT_TILE);
    const int64_t R = direct_resident_ctas();
    if (tiles >= 4 * R || ns <= DT_SPLIT_MIN_SRC) return {1, ns > 0 ? ns : 1};
    const int64_t smax = std::min<int64_t>(DT_SPLIT_MAX, ceil_div(ns, DT_SPLIT_MIN_SRC));
    DirectSplit best{1, ns};
    int64_t best_cost = INT64_MAX;
    for (int64_t s = 1; s <= smax; ++s) {
        const int64_t seg = ceil_div(ceil_div(ns, s), (int64_t)DT_CHUNK) * DT_CHUNK;
        const int64_t splits = ceil_div(ns, seg);
        const int64_t cost = ceil_div(tiles * splits, R) * seg;
        if (cost < best_cost) {
            best_cost = cost;
            best = {(int)splits, splits > 1 ? seg : ns};
        }
    }
    return best;
}

// Launch the plain direct sum on `stream` (no argument checks; used internally
// by the FMM's tol == 0 path and by the C-ABI entry below).  Split launches
// take their partial buffer from the context's arena.
pf_status launch_direct(pf_ctx *ctx, int64_t ns, const double *x, const double *y,
                        const double *g, int64_t nt, const double *xt, const double *yt,
                        double ksigmasqr, double *vx, double *vy, cudaStream_t stream,
                        bool cutoff) {
    if (nt == 0) return PF_OK;
    // cutoff: ksigmasqr is sigma^2 and only enters as the core term of r^2
    const pfd::GaussParams gp = pfd::make_gauss_params(cutoff ? 1.0 : ksigmasqr);
    constexpr int TPT = 2;
    const int64_t grid = ceil_div(nt, DT_TILE);
    if (grid > INT32_MAX) {
        set_error("pf_velocity_direct: too many targets (%lld)", (long long)nt);
        return PF_ERR_INVALID_ARG;
    }
    const DirectSplit sp = direct_split(ns, nt);
    float4 *part = nullptr;
    if (sp.splits > 1) {
        const size_t bytes = sizeof(float4) * (size_t)sp.splits * (size_t)nt;
        PF_TRY(arena_reserve(ctx, bytes + 256));
        part = static_cast<float4 *>(arena_take(ctx, bytes));
        if (!part) {
            set_error("pf_velocity_direct: scratch too small");
            return PF_ERR_OOM;
        }
    }
    if (cutoff) {
        k_direct_gauss<TPT, true>
            <<<dim3((unsigned)grid, (unsigned)sp.splits), DT_THREADS, 0, stream>>>(
                x, y, g, ns, sp.seg, xt, yt, nt, gp, vx, vy, part, (float)ksigmasqr);
    } else {
        k_direct_gauss<TPT><<<dim3((unsigned)grid, (unsigned)sp.splits), DT_THREADS, 0, stream>>>(
            x, y, g, ns, sp.seg, xt, yt, nt, gp, vx, vy, part);
    }
    PF_TRY(launch_status("k_direct_gauss"));
    if (!part) return PF_OK;
    k_direct_reduce<<<(unsigned)ceil_div(nt, DT_THREADS), DT_THREADS, 0, stream>>>(part, nt,
                                                                                 sp.splits, vx, vy);
    return launch_status("k_direct_reduce");
}

int direct_tile_targets() { return DT_THREADS * 2; }

pf_status launch_direct_batch(const DirectInstance *inst_dev, const int2 *items_dev, int n_items,
                              const int2 *reduce_items_dev, int n_reduce, int *counter_dev,
                              int grid, cudaStream_t st) {
    PF_CUDA_TRY(cudaMemsetAsync(counter_dev, 0, sizeof(int), st));
    if (n_items == 0) return PF_OK;
    k_direct_batch<<<grid, DT_THREADS, 0, st>>>(inst_dev, items_dev, n_items, counter_dev);
    PF_TRY(launch_status("k_direct_batch"));
    if (n_reduce == 0) return PF_OK;
    k_direct_reduce_batch<<<n_reduce, DT_THREADS, 0, st>>>(inst_dev, reduce_items_dev);
    return launch_status("k_direct_reduce_batch");
}

int direct_batch_grid(int num_sms) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_direct_batch, DT_THREADS, 0);
    if (per_sm < 1) per_sm = 1;
    return num_sms * per_sm;
}

}  // namespace pf

extern "C" pf_status pf_velocity_direct(pf_ctx *ctx, int64_t n_src, const double *x,
                                        const double *y, const double *g, int64_t n_tgt,
                                        const double *xt, const double *yt, double ksigmasqr,
                                        double *vx, double *vy, void *stream) {
    PF_RANGE("pf_velocity_direct");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_velocity_direct: NULL context");
    PF_CHECK_ARG(n_src >= 0 && n_tgt >= 0, "pf_velocity_direct: negative size");
    PF_CHECK_ARG(ksigmasqr > 0.0 && ksigmasqr < 1e300,
                 "pf_velocity_direct: ksigmasqr must be positive and finite (got %g)", ksigmasqr);
    PF_CHECK_ARG(n_src == 0 || (x && y && g), "pf_velocity_direct: NULL blob array");
    PF_CHECK_ARG(n_tgt == 0 || (xt && yt && vx && vy),
                 "pf_velocity_direct: NULL target/output array");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_tgt == 0) return PF_OK;
    if (n_src == 0) {
        PF_CUDA_TRY(cudaMemsetAsync(vx, 0, sizeof(double) * n_tgt, st));
        PF_CUDA_TRY(cudaMemsetAsync(vy, 0, sizeof(double) * n_tgt, st));
        return PF_OK;
    }
    return pf::launch_direct(ctx, n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, vx, vy, st);
}

extern "C" pf_status pf_velocity_direct_cutoff(pf_ctx *ctx, int64_t n_src, const double *x,
                                               const double *y, const double *g, int64_t n_tgt,
                                               const double *xt, const double *yt,
                                               double sigmasqr, double *vx, double *vy,
                                               void *stream) {
    PF_RANGE("pf_velocity_direct_cutoff");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_velocity_direct_cutoff: NULL context");
    PF_CHECK_ARG(n_src >= 0 && n_tgt >= 0, "pf_velocity_direct_cutoff: negative size");
    PF_CHECK_ARG(sigmasqr > 0.0 && sigmasqr < 1e30,
                 "pf_velocity_direct_cutoff: sigmasqr must be positive and finite (got %g)",
                 sigmasqr);
    PF_CHECK_ARG(n_src == 0 || (x && y && g), "pf_velocity_direct_cutoff: NULL blob array");
    PF_CHECK_ARG(n_tgt == 0 || (xt && yt && vx && vy),
                 "pf_velocity_direct_cutoff: NULL target/output array");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_tgt == 0) return PF_OK;
    if (n_src == 0) {
        PF_CUDA_TRY(cudaMemsetAsync(vx, 0, sizeof(double) * n_tgt, st));
        PF_CUDA_TRY(cudaMemsetAsync(vy, 0, sizeof(double) * n_tgt, st));
        return PF_OK;
    }
    return pf::launch_direct(ctx, n_src, x, y, g, n_tgt, xt, yt, sigmasqr, vx, vy, st, true);
}
