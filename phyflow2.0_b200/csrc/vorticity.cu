// vorticity.cu -- induced vorticity of Gaussian blobs by direct summation.
//
//   w_k = 1/(pi ksigmasqr) sum_m g_m exp(-r2/ksigmasqr),
//   r2 = dx^2 + dy^2 + 1e-12,  (dx, dy) = target_k - blob_m
//
// Replaces ww2parGauss_C_cpu (src/cpp/blobs/c/ww2parGauss_C/
// ww2parGauss_C_cpu.c:89-150) and its GPU twin, reached from
// _vorticity_direct_{cpu,gpu}_gauss (src/python/blobs/base/induced/
// _induced.py:702-963).  Same structure as the velocity direct sum
// (direct.cu): a CTA owns 512 targets (two per thread, packed f32x2), sources
// stream through shared memory as hi/lo float pairs, FP32 partial sums over 32
// sources fold into TwoSum-compensated (hi, lo) accumulators, and small sets
// cut the sources into segments (direct_split) reduced in segment order.
//
// The CUTOFF variant is the cutoff kernel's induced vorticity of
// ww2par_C_cpu (src/cpp/blobs/c/ww2par_C/ww2par_C_cpu.c:132-145) and its GPU
// twin (src/cpp/blobs/cuda/ww2par_gpu/ww2par_device.cu:59-70), as
// those compute it: w_k = 1/(2 pi) sum_m g_m / sqrt(r2 + sigma^2).
#include "direct_api.cuh"
#include "gauss_pair.cuh"

#include <algorithm>

namespace {

constexpr int VT_THREADS = 256;
constexpr int VT_CHUNK = 32;
constexpr int64_t VT_TILE = VT_THREADS * 2;
constexpr double INV_PI = 0.3183098861837907;  // 1/pi
constexpr double INV_2PI = 0.15915494309189535;  // 1/(2 pi)

// Two targets (packed) against one source: acc += g * 2^(r2 * c_t).
__device__ __forceinline__ void wpair2(const ulonglong2 &hi, const ulonglong2 &lo, pfd::f32x2 g2,
                                       pfd::f32x2 txh, pfd::f32x2 tyh, pfd::f32x2 txl,
                                       pfd::f32x2 tyl, const pfd::GaussParams2 &gp,
                                       pfd::f32x2 &acc) {
    const pfd::f32x2 dx = pfd::add2(pfd::sub2(txh, hi.x), pfd::sub2(txl, lo.x));
    const pfd::f32x2 dy = pfd::add2(pfd::sub2(tyh, hi.y), pfd::sub2(tyl, lo.y));
    const pfd::f32x2 r2 = pfd::fma2(dx, dx, pfd::fma2(dy, dy, gp.eps));
    float ta, tb;
    pfd::unpack2(pfd::mul2(r2, gp.c_t), ta, tb);
    acc = pfd::fma2(g2, pfd::pack2(pfd::ex2_approx(ta), pfd::ex2_approx(tb)), acc);
}

// Cutoff kernel: acc += g / sqrt(r2 + sigma^2), s2 = {sigma^2, sigma^2}.
__device__ __forceinline__ void wpair2_cutoff(const ulonglong2 &hi, const ulonglong2 &lo,
                                              pfd::f32x2 g2, pfd::f32x2 txh, pfd::f32x2 tyh,
                                              pfd::f32x2 txl, pfd::f32x2 tyl, pfd::f32x2 s2,
                                              pfd::f32x2 &acc) {
    const pfd::f32x2 dx = pfd::add2(pfd::sub2(txh, hi.x), pfd::sub2(txl, lo.x));
    const pfd::f32x2 dy = pfd::add2(pfd::sub2(tyh, hi.y), pfd::sub2(tyl, lo.y));
    const pfd::f32x2 r2 = pfd::fma2(dx, dx, pfd::fma2(dy, dy, s2));
    float ra, rb;
    pfd::unpack2(r2, ra, rb);
    acc = pfd::fma2(g2, pfd::pack2(pfd::rsqrt_approx(ra), pfd::rsqrt_approx(rb)), acc);
}

// w = (c1 * sum) / scale: Gauss c1 = 1/pi, scale = ksigmasqr; cutoff c1 =
// 1/(2 pi), scale = 1.
template <bool CUTOFF>
__global__ void __launch_bounds__(VT_THREADS)
k_vort_gauss(const double *__restrict__ xs, const double *__restrict__ ys,
             const double *__restrict__ gs, int64_t ns, int64_t seg,
             const double *__restrict__ xt, const double *__restrict__ yt, int64_t nt,
             pfd::GaussParams gp, double c1, double scale, float s2, double *__restrict__ w,
             float2 *__restrict__ part) {
    __shared__ ulonglong2 s_hi[VT_THREADS];  // {x_hi, x_hi}, {y_hi, y_hi}
    __shared__ ulonglong2 s_lo[VT_THREADS];  // {x_lo, x_lo}, {y_lo, y_lo}
    __shared__ unsigned long long s_g2[VT_THREADS];
    const int64_t s_begin = (int64_t)blockIdx.y * seg;
    const int64_t s_end = min(ns, s_begin + seg);
    const int64_t base = (int64_t)blockIdx.x * VT_TILE + threadIdx.x;
    float th[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int64_t i = base + (int64_t)j * VT_THREADS;
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
    float acc[4] = {0.f, 0.f, 0.f, 0.f};  // (hi, lo) of targets a and b
    for (int64_t t0 = s_begin; t0 < s_end; t0 += VT_THREADS) {
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
        const int nvalid = (int)min((int64_t)VT_THREADS, s_end - t0);
        for (int c0 = 0; c0 < nvalid; c0 += VT_CHUNK) {
            pfd::f32x2 p = 0ull;
#pragma unroll 4
            for (int k = 0; k < VT_CHUNK; ++k) {
                if (CUTOFF)
                    wpair2_cutoff(s_hi[c0 + k], s_lo[c0 + k], s_g2[c0 + k], txh, tyh, txl, tyl,
                                  s22, p);
                else
                    wpair2(s_hi[c0 + k], s_lo[c0 + k], s_g2[c0 + k], txh, tyh, txl, tyl, gp2, p);
            }
            float pa, pb;
            pfd::unpack2(p, pa, pb);
            pfd::comp_add(acc[0], acc[1], pa);
            pfd::comp_add(acc[2], acc[3], pb);
        }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int64_t i = base + (int64_t)j * VT_THREADS;
        if (i >= nt) continue;
        if (part)
            part[(int64_t)blockIdx.y * nt + i] = make_float2(acc[2 * j], acc[2 * j + 1]);
        else
            w[i] = (c1 * ((double)acc[2 * j] + (double)acc[2 * j + 1])) / scale;
    }
}

// w = (c1 * sum over segments of (hi + lo)) / scale, segments in order.
__global__ void __launch_bounds__(VT_THREADS)
k_vort_reduce(const float2 *__restrict__ part, int64_t nt, int splits, double c1, double scale,
              double *__restrict__ w) {
    const int64_t i = (int64_t)blockIdx.x * VT_THREADS + threadIdx.x;
    if (i >= nt) return;
    double s = 0.0;
    for (int k = 0; k < splits; ++k) {
        const float2 p = part[(int64_t)k * nt + i];
        s += (double)p.x + (double)p.y;
    }
    w[i] = (c1 * s) / scale;
}

}  // namespace

static pf_status vorticity_direct(pf_ctx *ctx, const char *name, int64_t n_src, const double *x,
                                  const double *y, const double *g, int64_t n_tgt,
                                  const double *xt, const double *yt, double param, double *w,
                                  void *stream, bool cutoff) {
    PF_CHECK_ARG(ctx != nullptr, "%s: NULL context", name);
    PF_CHECK_ARG(n_src >= 0 && n_tgt >= 0, "%s: negative size", name);
    PF_CHECK_ARG(param > 0.0 && param < (cutoff ? 1e30 : 1e300),
                 "%s: %s must be positive and finite (got %g)", name,
                 cutoff ? "sigmasqr" : "ksigmasqr", param);
    PF_CHECK_ARG(n_src == 0 || (x && y && g), "%s: NULL blob array", name);
    PF_CHECK_ARG(n_tgt == 0 || (xt && yt && w), "%s: NULL target/output array", name);
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_tgt == 0) return PF_OK;
    if (n_src == 0) {
        PF_CUDA_TRY(cudaMemsetAsync(w, 0, sizeof(double) * n_tgt, st));
        return PF_OK;
    }
    const int64_t grid = pf::ceil_div(n_tgt, VT_TILE);
    PF_CHECK_ARG(grid <= INT32_MAX, "%s: too many targets (%lld)", name, (long long)n_tgt);
    const pfd::GaussParams gp = pfd::make_gauss_params(cutoff ? 1.0 : param);
    const double c1 = cutoff ? INV_2PI : INV_PI, scale = cutoff ? 1.0 : param;
    const float s2 = cutoff ? (float)param : 0.f;
    const pf::DirectSplit sp = pf::direct_split(n_src, n_tgt);
    float2 *part = nullptr;
    if (sp.splits > 1) {
        const size_t bytes = sizeof(float2) * (size_t)sp.splits * (size_t)n_tgt;
        PF_TRY(pf::arena_reserve(ctx, bytes + 256));
        part = static_cast<float2 *>(pf::arena_take(ctx, bytes));
        if (!part) {
            pf::set_error("%s: scratch too small", name);
            return PF_ERR_OOM;
        }
    }
    const dim3 grd((unsigned)grid, (unsigned)sp.splits);
    if (cutoff)
        k_vort_gauss<true><<<grd, VT_THREADS, 0, st>>>(x, y, g, n_src, sp.seg, xt, yt, n_tgt, gp,
                                                       c1, scale, s2, w, part);
    else
        k_vort_gauss<false><<<grd, VT_THREADS, 0, st>>>(x, y, g, n_src, sp.seg, xt, yt, n_tgt, gp,
                                                        c1, scale, s2, w, part);
    PF_TRY(pf::launch_status("k_vort_gauss"));
    if (!part) return PF_OK;
    k_vort_reduce<<<(unsigned)pf::ceil_div(n_tgt, VT_THREADS), VT_THREADS, 0, st>>>(
        part, n_tgt, sp.splits, c1, scale, w);
    return pf::launch_status("k_vort_reduce");
}

extern "C" pf_status pf_vorticity_direct(pf_ctx *ctx, int64_t n_src, const double *x,
                                         const double *y, const double *g, int64_t n_tgt,
                                         const double *xt, const double *yt, double ksigmasqr,
                                         double *w, void *stream) {
    PF_RANGE("pf_vorticity_direct");
    pf::clear_error();
    return vorticity_direct(ctx, "pf_vorticity_direct", n_src, x, y, g, n_tgt, xt, yt, ksigmasqr,
                            w, stream, false);
}

extern "C" pf_status pf_vorticity_direct_cutoff(pf_ctx *ctx, int64_t n_src, const double *x,
                                                const double *y, const double *g, int64_t n_tgt,
                                                const double *xt, const double *yt,
                                                double sigmasqr, double *w, void *stream) {
    PF_RANGE("pf_vorticity_direct_cutoff");
    pf::clear_error();
    return vorticity_direct(ctx, "pf_vorticity_direct_cutoff", n_src, x, y, g, n_tgt, xt, yt,
                            sigmasqr, w, stream, true);
}
