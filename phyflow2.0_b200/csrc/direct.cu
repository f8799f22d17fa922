// direct.cu -- Gaussian-blob Biot-Savart velocity by direct summation.
//
// One simulation per launch (the plain path).  Each CTA owns DT_THREADS*TPT
// targets (TPT per thread, coalesced); all CTAs stream the whole source set
// through shared memory in tiles of DT_THREADS blobs, converted on load from
// FP64 to hi/lo float pairs (so no scratch buffer is needed).  Per thread the
// pair sums run in FP32 over chunks of 32 sources and are folded into a
// TwoSum-compensated (hi, lo) accumulator after each chunk.
//
// Replaces vv2par_kernel (src/cpp/blobs/cuda/vv2parGauss_gpu/
// vv2parGauss_device.cu:107-162: FP64, one target per thread, 2 exp per pair,
// targets padded to a multiple of the block size by the Python caller).
#include "direct_api.cuh"
#include "gauss_pair.cuh"

namespace {

constexpr int DT_THREADS = 256;
constexpr int DT_CHUNK = 32;
constexpr double INV_2PI = 0.15915494309189535;  // 0.5/pi

// One CTA computes the 2*DT_THREADS targets of tile `tile`: each thread owns
// targets base and base + DT_THREADS and evaluates both against every source
// with the packed f32x2 pair arithmetic (gauss_pair.cuh).
__device__ __forceinline__ void direct_tile(const double *__restrict__ xs,
                                            const double *__restrict__ ys,
                                            const double *__restrict__ gs, int64_t ns,
                                            const double *__restrict__ xt,
                                            const double *__restrict__ yt, int64_t nt,
                                            const pfd::GaussParams &gp, double *__restrict__ vx,
                                            double *__restrict__ vy, int64_t tile,
                                            ulonglong2 *s_hi, ulonglong2 *s_lo,
                                            unsigned long long *s_g2) {
    const int64_t base = tile * (DT_THREADS * 2) + threadIdx.x;
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
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};

    for (int64_t t0 = 0; t0 < ns; t0 += DT_THREADS) {
        const int64_t s = t0 + threadIdx.x;
        double x = 0.0, y = 0.0, g = 0.0;  // padding blobs carry g = 0
        if (s < ns) {
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
        const int nvalid = (int)min((int64_t)DT_THREADS, ns - t0);
        for (int c0 = 0; c0 < nvalid; c0 += DT_CHUNK) {
            pfd::f32x2 nx = 0ull, ny = 0ull;
#pragma unroll 4
            for (int k = 0; k < DT_CHUNK; ++k)
                pfd::pair2(s_hi[c0 + k], s_lo[c0 + k], s_g2[c0 + k], txh, tyh, txl, tyl, gp2, nx,
                           ny);
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
        if (i < nt) {
            vx[i] = INV_2PI * ((double)acc[4 * j] + (double)acc[4 * j + 1]);
            vy[i] = INV_2PI * ((double)acc[4 * j + 2] + (double)acc[4 * j + 3]);
        }
    }
}

template <int TPT>
__global__ void __launch_bounds__(DT_THREADS)
k_direct_gauss(const double *__restrict__ xs, const double *__restrict__ ys,
               const double *__restrict__ gs, int64_t ns, const double *__restrict__ xt,
               const double *__restrict__ yt, int64_t nt, pfd::GaussParams gp,
               double *__restrict__ vx, double *__restrict__ vy) {
    static_assert(TPT == 2, "two targets per thread (packed pairs)");
    __shared__ ulonglong2 s_hi[DT_THREADS];  // {x_hi, x_hi}, {y_hi, y_hi}
    __shared__ ulonglong2 s_lo[DT_THREADS];  // {x_lo, x_lo}, {y_lo, y_lo}
    __shared__ unsigned long long s_g2[DT_THREADS];
    direct_tile(xs, ys, gs, ns, xt, yt, nt, gp, vx, vy, blockIdx.x, s_hi, s_lo, s_g2);
}

// Persistent batched direct sum: CTAs take (instance, target tile) items from
// a device counter until the list is exhausted.  Items are ordered by cost,
// largest first; each item is computed by one CTA, so results do not depend
// on which CTA takes it.
__global__ void __launch_bounds__(DT_THREADS)
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
        direct_tile(d.x, d.y, d.g, d.n, d.xt, d.yt, d.nt, d.gp, d.vx, d.vy, w.y, s_hi, s_lo, s_g2);
    }
}

}  // namespace

namespace pf {

// Launch the plain direct sum on `stream` (no argument checks; used internally
// by the FMM's tol == 0 path and by the C-ABI entry below).
pf_status launch_direct(int64_t ns, const double *x, const double *y, const double *g,
                        int64_t nt, const double *xt, const double *yt, double ksigmasqr,
                        double *vx, double *vy, cudaStream_t stream) {
    if (nt == 0) return PF_OK;
    const pfd::GaussParams gp = pfd::make_gauss_params(ksigmasqr);
    constexpr int TPT = 2;
    const int64_t per = DT_THREADS * TPT;
    const int64_t grid = ceil_div(nt, per);
    if (grid > INT32_MAX) {
        set_error("pf_velocity_direct: too many targets (%lld)", (long long)nt);
        return PF_ERR_INVALID_ARG;
    }
    k_direct_gauss<TPT><<<(unsigned)grid, DT_THREADS, 0, stream>>>(x, y, g, ns, xt, yt, nt, gp,
                                                                   vx, vy);
    return launch_status("k_direct_gauss");
}

int direct_tile_targets() { return DT_THREADS * 2; }

pf_status launch_direct_batch(const DirectInstance *inst_dev, const int2 *items_dev, int n_items,
                              int *counter_dev, int grid, cudaStream_t st) {
    PF_CUDA_TRY(cudaMemsetAsync(counter_dev, 0, sizeof(int), st));
    if (n_items == 0) return PF_OK;
    k_direct_batch<<<grid, DT_THREADS, 0, st>>>(inst_dev, items_dev, n_items, counter_dev);
    return launch_status("k_direct_batch");
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
    return pf::launch_direct(n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, vx, vy, st);
}
