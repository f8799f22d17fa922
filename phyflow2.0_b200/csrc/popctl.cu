// popctl.cu -- PopulationControl on the device.
//
// Reference (src/python/blobs/base/regrid/_regridding.py:316-330): flag the
// blobs with |g| < thr; if the flagged circulation sum(|g|) is not below
// gThresholdGlobal, divide thr by 10 and flag again; finally keep the
// unflagged blobs in their original order.
//
// Here the decade loop is evaluated without host round trips.  With
// thr_k = thr / 10 / ... / 10 (k divisions, rounded as the reference's loop)
// and loss_k = sum of |g| over |g| < thr_k, one launch of k_pc_loss computes
// loss_k for PC_DECADES consecutive k at once (each thread keeps PC_DECADES
// FP64 partial sums), and the last CTA to finish sums the per-CTA partials in
// CTA order and picks the first k with loss_k < gThresholdGlobal.  Because
// loss_k <= n * thr_k, the decision is reached by the first k with
// 2 n thr_k < gThresholdGlobal, which bounds the number of launches (one for
// every practical threshold pair; later launches return at once).  The grid
// and the reduction order are fixed, so the decision is deterministic.  The
// sums are FP64 in a different order from numpy's pairwise sum, so a loss
// within rounding of gThresholdGlobal could be decided differently.
//
// The kept blobs are then compacted in input order: keep flags, exclusive
// scan, scatter.
#include "popctl.cuh"
#include "scan.cuh"

#include <cmath>

namespace {

constexpr int PC_DECADES = 16;
constexpr int PC_THREADS = 256;
constexpr int PC_BLOCKS = 592;

struct Decades {
    double t[PC_DECADES];
    int32_t base;
    int32_t last;
};

__global__ void __launch_bounds__(PC_THREADS)
k_pc_loss(int64_t n, const int64_t *__restrict__ n_dev, const double *__restrict__ g,
          const int32_t *__restrict__ flag, Decades d, double limit, double *__restrict__ part,
          pf::PcState *__restrict__ st) {
    __shared__ double s_w[PC_THREADS / 32][PC_DECADES];
    __shared__ double s_tot[PC_DECADES];
    __shared__ int s_last;
    if (st->decided) return;  // decided by an earlier launch: same value for every CTA
    if (n_dev) n = *n_dev;    // the value count known on the device only (n bounds it)
    const int64_t chunk = (n + PC_BLOCKS - 1) / PC_BLOCKS;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = min(n, lo + chunk);
    double acc[PC_DECADES];
#pragma unroll
    for (int k = 0; k < PC_DECADES; ++k) acc[k] = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += PC_THREADS) {
        if (flag && !flag[i]) continue;
        const double v = fabs(g[i]);
#pragma unroll
        for (int k = 0; k < PC_DECADES; ++k)
            if (v < d.t[k]) acc[k] += v;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < PC_DECADES; ++k) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_w[wid][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < PC_DECADES) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < PC_THREADS / 32; ++w) s += s_w[w][threadIdx.x];
        part[(int64_t)blockIdx.x * PC_DECADES + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(&st->done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x < PC_DECADES) {
        double s = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(&part[b * PC_DECADES + threadIdx.x]);
        s_tot[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < PC_DECADES; ++k) {
            if (s_tot[k] < limit) {
                st->thr = d.t[k];
                st->k = d.base + k;
                st->decided = 1;
                break;
            }
        }
        if (!st->decided && d.last) {  // not reached (loss_k <= n thr_k bound); keeps st defined
            st->thr = d.t[PC_DECADES - 1];
            st->k = d.base + PC_DECADES - 1;
            st->decided = 1;
        }
        st->done = 0u;
    }
}

__global__ void __launch_bounds__(PC_THREADS)
k_pc_flags(int64_t n, const double *__restrict__ g, const int32_t *flag_in,
           const pf::PcState *__restrict__ st, int32_t *flag_out) {
    const int64_t i = (int64_t)blockIdx.x * PC_THREADS + threadIdx.x;
    if (i >= n) return;
    const int keep_in = flag_in ? (flag_in[i] != 0) : 1;
    flag_out[i] = keep_in && !(fabs(g[i]) < st->thr);
}

__global__ void __launch_bounds__(PC_THREADS)
k_pc_scatter(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
             const double *__restrict__ g, const int32_t *__restrict__ flag,
             const int32_t *__restrict__ slot, double *__restrict__ xo, double *__restrict__ yo,
             double *__restrict__ go) {
    const int64_t i = (int64_t)blockIdx.x * PC_THREADS + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const int64_t p = slot[i];
    xo[p] = x[i];
    yo[p] = y[i];
    go[p] = g[i];
}

__global__ void k_pc_finish(const int32_t *__restrict__ total, const pf::PcState *__restrict__ st,
                            int64_t *__restrict__ n_out_dev, double *__restrict__ thr_dev) {
    *n_out_dev = *total;
    if (thr_dev) *thr_dev = st->thr;
}

}  // namespace

namespace pf {

pf_status popctl_check(double thr_local, double thr_global, const char *who) {
    PF_CHECK_ARG(std::isfinite(thr_local), "%s: gThresholdLocal must be finite", who);
    // a limit <= 0 (or NaN) is never met: the reference's loop would not end
    PF_CHECK_ARG(std::isfinite(thr_global) && thr_global > 0.0,
                 "%s: gThresholdGlobal must be positive and finite", who);
    return PF_OK;
}

size_t popctl_scratch_bytes() {
    return align256(sizeof(double) * PC_BLOCKS * PC_DECADES) + 256;
}

pf_status popctl_decide(Bump &sc, int64_t n, const double *g, const int32_t *flag,
                        const PopCtlArgs &pc, cudaStream_t st, const int64_t *n_dev) {
    double *part = (double *)sc.take(sizeof(double) * PC_BLOCKS * PC_DECADES);
    if (!part) {
        set_error("population control: scratch too small");
        return PF_ERR_OOM;
    }
    // number of decades that can be needed (see the file comment)
    int kmax = 0;
    for (double t = pc.thr_local; t > 0.0 && !(2.0 * (double)n * t < pc.thr_global); t /= 10.0)
        ++kmax;
    const int launches = kmax / PC_DECADES + 1;
    PF_CUDA_TRY(cudaMemsetAsync(pc.state, 0, sizeof(PcState), st));
    double t = pc.thr_local;
    for (int L = 0; L < launches; ++L) {
        Decades d;
        for (int j = 0; j < PC_DECADES; ++j) {
            d.t[j] = t;
            t /= 10.0;  // the reference's `wThreshold /= 10.0`
        }
        d.base = L * PC_DECADES;
        d.last = (L == launches - 1);
        k_pc_loss<<<PC_BLOCKS, PC_THREADS, 0, st>>>(n, n_dev, g, flag, d, pc.thr_global, part,
                                                    pc.state);
        PF_TRY(launch_status("k_pc_loss"));
    }
    return PF_OK;
}

pf_status popctl_flags(int64_t n, const double *g, const int32_t *flag_in, const PcState *state,
                       int32_t *flag_out, cudaStream_t st) {
    if (n == 0) return PF_OK;
    k_pc_flags<<<(unsigned)ceil_div(n, PC_THREADS), PC_THREADS, 0, st>>>(n, g, flag_in, state,
                                                                          flag_out);
    return launch_status("k_pc_flags");
}

}  // namespace pf

extern "C" pf_status pf_population_control(pf_ctx *ctx, int64_t n, const double *x,
                                           const double *y, const double *g,
                                           double g_threshold_local, double g_threshold_global,
                                           double *x_out, double *y_out, double *g_out,
                                           int64_t *n_out_dev, double *threshold_dev,
                                           void *stream) {
    PF_RANGE("pf_population_control");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_population_control: NULL context");
    PF_CHECK_ARG(n >= 0 && n < ((int64_t)1 << 31), "pf_population_control: n = %lld outside [0, 2^31)",
                 (long long)n);
    PF_TRY(pf::popctl_check(g_threshold_local, g_threshold_global, "pf_population_control"));
    PF_CHECK_ARG(n == 0 || (x && y && g && x_out && y_out && g_out),
                 "pf_population_control: NULL array");
    PF_CHECK_ARG(n_out_dev != nullptr, "pf_population_control: n_out_dev is NULL");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t need = 2 * pf::align256(4 * (size_t)n) +
                        pf::align256(4 * pf::scan_tmp_ints(n > 0 ? n : 1)) +
                        pf::popctl_scratch_bytes() + 3 * pf::align256(64) + 1024;
    PF_TRY(pf::arena_reserve(ctx, need));
    pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
    pf::PcState *state = (pf::PcState *)sc.take(sizeof(pf::PcState));
    int32_t *total = (int32_t *)sc.take(16);
    int32_t *flag = (int32_t *)sc.take(4 * (size_t)n);
    int32_t *slot = (int32_t *)sc.take(4 * (size_t)n);
    int32_t *tmp = (int32_t *)sc.take(4 * pf::scan_tmp_ints(n > 0 ? n : 1));
    if (!state || !total || (n > 0 && (!flag || !slot)) || !tmp) {
        pf::set_error("pf_population_control: scratch too small");
        return PF_ERR_OOM;
    }
    pf::PopCtlArgs pc{g_threshold_local, g_threshold_global, state};
    PF_TRY(pf::popctl_decide(sc, n, g, nullptr, pc, st));
    PF_TRY(pf::popctl_flags(n, g, nullptr, state, flag, st));
    PF_TRY(pf::exclusive_scan_i32(flag, slot, n, tmp, total, st));
    if (n > 0) {
        k_pc_scatter<<<(unsigned)pf::ceil_div(n, PC_THREADS), PC_THREADS, 0, st>>>(
            n, x, y, g, flag, slot, x_out, y_out, g_out);
        PF_TRY(pf::launch_status("k_pc_scatter"));
    }
    k_pc_finish<<<1, 1, 0, st>>>(total, state, n_out_dev, threshold_dev);
    return pf::launch_status("k_pc_finish");
}
