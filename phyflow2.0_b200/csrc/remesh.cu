// remesh.cu -- M4' remesh (pHyFlow Regrid) on a dense lattice window.
//
// Pipeline (all FP64 values, integer cell work bit-exact):
//   1. k_rm_extent : window-left lattice index of every blob,
//        xl = ceil(((x - xb0) - 2h) + 0.5h) / h) - 1     (_regridding.py:157-158)
//      with the same operation order as numpy (IEEE, no FMA contraction:
//      2h and 0.5h are formed on the host); min/max over blobs -> extent.
//   [host reads the extent: one stream sync]
//   2. k_rm_count  : counting sort of blobs by base cell (xl, yl), base
//      cells in ix-major order; rank of a blob in its cell from atomicAdd.
//   3. scan of the per-cell counts -> cell starts.
//   4. k_rm_place  : blob index -> its slot.
//   5. k_rm_order  : per base cell, order its blobs by input index (so every
//      sum below has a fixed order, independent of atomic timing) and write
//      the blob data in that order (x/h, y/h, g): a cell-sorted copy.
//   6. k_rm_gather : one thread per output cell (ix, iy); it sums, in fixed
//      order, the M4'(ux) M4'(uy) g contributions of the blobs of the 16 base
//      cells whose windows cover it (_regridding.py:183-184, weights of
//      _interpolation_kernels_1d.cpp:75-89), and flags cells touched by at
//      least one window (explicit zeros are kept, like the CSR sum of the
//      reference, _regridding.py:200-202).
//   7. scan of the flags -> output slots, in (ix, iy) order.
//   8. k_rm_emit   : x = ix*h + 0.5h + xb0 (same order as :217-218), g, ix, iy.
//   [host reads the count: second stream sync]
// No floating-point atomics: each output value is produced by one thread.
#include <cmath>
#include <cstring>

#include "scan.cuh"

namespace {

constexpr int RM_THREADS = 256;

struct Extent {
    int32_t ixmin, ixmax, iymin, iymax;
    int32_t bad;  // 1: NaN/Inf coordinate, 2: index outside +-2^30
    int32_t pad[3];
};

__device__ __forceinline__ int64_t left_index(double x, double b0, double h2, double h05,
                                              double h) {
    // ((x - b0) - 2h) + 0.5h, then / h, ceil, -1 ; each op rounded separately
    double t = __dadd_rn(__dsub_rn(__dsub_rn(x, b0), h2), h05);
    double q = __ddiv_rn(t, h);
    return (int64_t)ceil(q) - 1;
}

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

__global__ void k_rm_extent_init(Extent *e) {
    e->ixmin = INT32_MAX;
    e->iymin = INT32_MAX;
    e->ixmax = INT32_MIN;
    e->iymax = INT32_MIN;
    e->bad = 0;
}

__device__ __forceinline__ int warp_min(int v) {
    for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max(int v) {
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

constexpr int64_t IDX_LIMIT = (int64_t)1 << 30;

__global__ void __launch_bounds__(RM_THREADS)
k_rm_extent(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double xb0,
            double yb0, double h2, double h05, double h, Extent *e) {
    int mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN, bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * RM_THREADS) {
        const double xi = x[i], yi = y[i];
        if (!finite_d(xi) || !finite_d(yi)) {
            bad |= 1;
            continue;
        }
        const int64_t a = left_index(xi, xb0, h2, h05, h);
        const int64_t b = left_index(yi, yb0, h2, h05, h);
        if (a < -IDX_LIMIT || a > IDX_LIMIT || b < -IDX_LIMIT || b > IDX_LIMIT) {
            bad |= 2;
            continue;
        }
        mnx = min(mnx, (int)a);
        mxx = max(mxx, (int)a);
        mny = min(mny, (int)b);
        mxy = max(mxy, (int)b);
    }
    mnx = warp_min(mnx);
    mxx = warp_max(mxx);
    mny = warp_min(mny);
    mxy = warp_max(mxy);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        if (mnx != INT32_MAX) {
            atomicMin(&e->ixmin, mnx);
            atomicMax(&e->ixmax, mxx);
            atomicMin(&e->iymin, mny);
            atomicMax(&e->iymax, mxy);
        }
        if (bad) atomicOr(&e->bad, bad);
    }
}

// base cell grid: bx in [0, nbx), by in [0, nby), id = bx*nby + by
__global__ void __launch_bounds__(RM_THREADS)
k_rm_count(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double xb0,
           double yb0, double h2, double h05, double h, int32_t ixmin, int32_t iymin, int64_t nby,
           int32_t *__restrict__ cell, int32_t *__restrict__ rank, int32_t *__restrict__ count) {
    const int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (i >= n) return;
    const int64_t a = left_index(x[i], xb0, h2, h05, h) - ixmin;
    const int64_t b = left_index(y[i], yb0, h2, h05, h) - iymin;
    const int32_t c = (int32_t)(a * nby + b);
    cell[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

__global__ void __launch_bounds__(RM_THREADS)
k_rm_place(int64_t n, const int32_t *__restrict__ cell, const int32_t *__restrict__ rank,
           const int32_t *__restrict__ start, int32_t *__restrict__ perm) {
    const int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (i >= n) return;
    perm[start[cell[i]] + rank[i]] = (int32_t)i;
}

__global__ void __launch_bounds__(RM_THREADS)
k_rm_order(int64_t ncell, const int32_t *__restrict__ start, const int32_t *__restrict__ count,
           int32_t *__restrict__ perm, const double *__restrict__ x, const double *__restrict__ y,
           const double *__restrict__ g, double h, double *__restrict__ sxh,
           double *__restrict__ syh, double *__restrict__ sg) {
    const int64_t c = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (c >= ncell) return;
    const int cnt = count[c];
    if (cnt == 0) return;
    const int s0 = start[c];
    // insertion sort of the cell's blob indices (cells hold a few blobs)
    for (int k = 1; k < cnt; ++k) {
        const int32_t v = perm[s0 + k];
        int j = k - 1;
        while (j >= 0 && perm[s0 + j] > v) {
            perm[s0 + j + 1] = perm[s0 + j];
            --j;
        }
        perm[s0 + j + 1] = v;
    }
    for (int k = 0; k < cnt; ++k) {
        const int32_t i = perm[s0 + k];
        sxh[s0 + k] = __ddiv_rn(x[i], h);
        syh[s0 + k] = __ddiv_rn(y[i], h);
        sg[s0 + k] = g[i];
    }
}

// M4' weight with the Wee term: branch structure of
// _interpolation_kernels_1d.cpp:77-88 (open interval (1,2), then [0,1), else 0)
__device__ __forceinline__ double m4p(double u, double c2) {
    const double a = fabs(u);
    if (a > 1.0 && a < 2.0) {
        const double t = 2.0 - a;
        const double t2 = t * t;
        return 0.5 * t2 * (1.0 - a) - c2 * t2 * (1.0 - 2.0 * a);
    } else if (a < 1.0) {
        const double a2 = u * u;
        const double a3 = a * a * a;
        return 1.0 - 2.5 * a2 + 1.5 * a3 - c2 * (2.0 - 9.0 * a2 + 6.0 * a3);
    }
    return 0.0;
}

// Output cell grid: ox in [0, nbx+3), oy in [0, nby+3); lattice index
// ix = ixmin + ox.  A base cell (bx, by) covers ox in bx..bx+3, oy in by..by+3.
__global__ void __launch_bounds__(RM_THREADS)
k_rm_gather(int64_t nbx, int64_t nby, int32_t ixmin, int32_t iymin, double qx0, double qy0,
            double c2, const int32_t *__restrict__ start, const int32_t *__restrict__ count,
            const double *__restrict__ sxh, const double *__restrict__ syh,
            const double *__restrict__ sg, double *__restrict__ acc, int32_t *__restrict__ flag) {
    const int64_t noy = nby + 3;
    const int64_t cid = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (cid >= (nbx + 3) * noy) return;
    const int64_t ox = cid / noy, oy = cid - ox * noy;
    // numpy: (ix + 0.5) + xb0/h - x/h  with ix the absolute lattice index
    const double px = ((double)(ixmin + ox) + 0.5) + qx0;
    const double py = ((double)(iymin + oy) + 0.5) + qy0;
    double sum = 0.0;
    int touched = 0;
    // window offsets: x offset a = ox - bx fastest in the reference numbering,
    // but each output cell sums over (a, b) in a fixed order of its own
#pragma unroll 1
    for (int b = 0; b < 4; ++b) {
        const int64_t by = oy - b;
        if (by < 0 || by >= nby) continue;
#pragma unroll 1
        for (int a = 0; a < 4; ++a) {
            const int64_t bx = ox - a;
            if (bx < 0 || bx >= nbx) continue;
            const int64_t bc = bx * nby + by;
            const int cnt = count[bc];
            if (cnt == 0) continue;
            touched = 1;
            const int s0 = start[bc];
            for (int k = 0; k < cnt; ++k) {
                const double wx = m4p(__dsub_rn(px, sxh[s0 + k]), c2);
                const double wy = m4p(__dsub_rn(py, syh[s0 + k]), c2);
                sum += (wx * wy) * sg[s0 + k];
            }
        }
    }
    acc[cid] = sum;
    flag[cid] = touched;
}

__global__ void __launch_bounds__(RM_THREADS)
k_rm_emit(int64_t ncell, int64_t noy, int32_t ixmin, int32_t iymin, double h, double h05,
          double xb0, double yb0, const int32_t *__restrict__ flag,
          const int32_t *__restrict__ slot, const double *__restrict__ acc,
          const int32_t *__restrict__ total, int64_t capacity, double *__restrict__ xo,
          double *__restrict__ yo, double *__restrict__ go, int64_t *__restrict__ ixo,
          int64_t *__restrict__ iyo) {
    const int64_t cid = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (cid >= ncell) return;
    if ((int64_t)(*total) > capacity) return;  // capacity error: write nothing
    if (!flag[cid]) return;
    const int64_t ox = cid / noy, oy = cid - ox * noy;
    const int64_t ix = ixmin + ox, iy = iymin + oy;
    const int64_t p = slot[cid];
    // (ix*h + 0.5h) + xb0, each operation rounded (no FMA)
    xo[p] = __dadd_rn(__dadd_rn(__dmul_rn((double)ix, h), h05), xb0);
    yo[p] = __dadd_rn(__dadd_rn(__dmul_rn((double)iy, h), h05), yb0);
    go[p] = acc[cid];
    if (ixo) ixo[p] = ix;
    if (iyo) iyo[p] = iy;
}

}  // namespace

namespace pf {

// Dense-window limit: base cells <= max(2^26, 64 n).  Beyond it the blob set
// is too sparse for a dense lattice window and the call is rejected.
static int64_t dense_cell_limit(int64_t n) {
    int64_t a = (int64_t)1 << 26;
    int64_t b = 64 * n;
    int64_t lim = a > b ? a : b;
    return lim < ((int64_t)1 << 30) ? lim : ((int64_t)1 << 30);
}

}  // namespace pf

extern "C" pf_status pf_remesh(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                               const double *g, double h, double xb0, double yb0, double c,
                               int64_t capacity, double *x_out, double *y_out, double *g_out,
                               int64_t *ix_out, int64_t *iy_out, int64_t *n_out, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_remesh: NULL context");
    PF_CHECK_ARG(n_out != nullptr, "pf_remesh: n_out is NULL");
    *n_out = 0;
    PF_CHECK_ARG(n >= 0 && n < ((int64_t)1 << 31), "pf_remesh: n = %lld outside [0, 2^31)",
                 (long long)n);
    PF_CHECK_ARG(std::isfinite(h) && h > 0.0, "pf_remesh: h must be positive and finite");
    PF_CHECK_ARG(std::isfinite(xb0) && std::isfinite(yb0) && std::isfinite(c),
                 "pf_remesh: bounds and c must be finite");
    PF_CHECK_ARG(n == 0 || (x && y && g), "pf_remesh: NULL input array");
    PF_CHECK_ARG(capacity >= 0, "pf_remesh: negative capacity");
    if (n == 0) return PF_OK;
    PF_CHECK_ARG(capacity == 0 || (x_out && y_out && g_out), "pf_remesh: NULL output array");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    const double h2 = 2.0 * h, h05 = 0.5 * h;
    // scratch phase 1: the extent record
    PF_TRY(pf::arena_reserve(ctx, 4096));
    Extent *ext = static_cast<Extent *>(pf::arena_take(ctx, sizeof(Extent)));
    k_rm_extent_init<<<1, 1, 0, st>>>(ext);
    PF_TRY(pf::launch_status("k_rm_extent_init"));
    {
        int64_t grid = pf::ceil_div(n, RM_THREADS);
        int64_t cap = (int64_t)ctx->num_sms * 8;
        if (grid > cap) grid = cap;
        k_rm_extent<<<(unsigned)grid, RM_THREADS, 0, st>>>(x, y, n, xb0, yb0, h2, h05, h, ext);
        PF_TRY(pf::launch_status("k_rm_extent"));
    }
    Extent he;
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->host_small, ext, sizeof(Extent), cudaMemcpyDeviceToHost, st));
    PF_CUDA_TRY(cudaStreamSynchronize(st));
    memcpy(&he, ctx->host_small, sizeof(Extent));
    if (he.bad & 1) {
        pf::set_error("pf_remesh: NaN or Inf blob coordinate");
        return PF_ERR_NAN_INPUT;
    }
    if (he.bad & 2) {
        pf::set_error("pf_remesh: blob lattice index beyond +-2^30 (coordinates far from bounds)");
        return PF_ERR_INVALID_ARG;
    }
    const int64_t nbx = (int64_t)he.ixmax - he.ixmin + 1;
    const int64_t nby = (int64_t)he.iymax - he.iymin + 1;
    const int64_t nbase = nbx * nby;
    const int64_t ncell = (nbx + 3) * (nby + 3);
    if (nbase > pf::dense_cell_limit(n) || ncell >= ((int64_t)1 << 31)) {
        pf::set_error("pf_remesh: lattice window %lld x %lld is too large for %lld blobs",
                      (long long)nbx, (long long)nby, (long long)n);
        return PF_ERR_INVALID_ARG;
    }

    // scratch phase 2
    const size_t need = pf::align256(sizeof(Extent)) + 2 * pf::align256(4 * n) /* cell, rank */ +
                        pf::align256(4 * n) /* perm */ + 3 * pf::align256(8 * n) /* sorted */ +
                        2 * pf::align256(4 * nbase) /* count, start */ +
                        pf::align256(8 * ncell) /* acc */ + 2 * pf::align256(4 * ncell) /* flag, slot */ +
                        pf::align256(4 * pf::scan_tmp_ints(ncell > nbase ? ncell : nbase)) +
                        pf::align256(16) + 4096;
    PF_TRY(pf::arena_reserve(ctx, need));
    (void)pf::arena_take(ctx, sizeof(Extent));
    int32_t *cell = static_cast<int32_t *>(pf::arena_take(ctx, 4 * n));
    int32_t *rank = static_cast<int32_t *>(pf::arena_take(ctx, 4 * n));
    int32_t *perm = static_cast<int32_t *>(pf::arena_take(ctx, 4 * n));
    double *sxh = static_cast<double *>(pf::arena_take(ctx, 8 * n));
    double *syh = static_cast<double *>(pf::arena_take(ctx, 8 * n));
    double *sg = static_cast<double *>(pf::arena_take(ctx, 8 * n));
    int32_t *count = static_cast<int32_t *>(pf::arena_take(ctx, 4 * nbase));
    int32_t *start = static_cast<int32_t *>(pf::arena_take(ctx, 4 * nbase));
    double *acc = static_cast<double *>(pf::arena_take(ctx, 8 * ncell));
    int32_t *flag = static_cast<int32_t *>(pf::arena_take(ctx, 4 * ncell));
    int32_t *slot = static_cast<int32_t *>(pf::arena_take(ctx, 4 * ncell));
    int32_t *tmp = static_cast<int32_t *>(
        pf::arena_take(ctx, 4 * pf::scan_tmp_ints(ncell > nbase ? ncell : nbase)));
    int32_t *total = static_cast<int32_t *>(pf::arena_take(ctx, 16));
    if (!total) {
        pf::set_error("pf_remesh: internal scratch layout error");
        return PF_ERR_OOM;
    }

    const unsigned gn = (unsigned)pf::ceil_div(n, RM_THREADS);
    PF_CUDA_TRY(cudaMemsetAsync(count, 0, 4 * nbase, st));
    k_rm_count<<<gn, RM_THREADS, 0, st>>>(x, y, n, xb0, yb0, h2, h05, h, he.ixmin, he.iymin, nby,
                                          cell, rank, count);
    PF_TRY(pf::launch_status("k_rm_count"));
    PF_TRY(pf::exclusive_scan_i32(count, start, nbase, tmp, nullptr, st));
    k_rm_place<<<gn, RM_THREADS, 0, st>>>(n, cell, rank, start, perm);
    PF_TRY(pf::launch_status("k_rm_place"));
    k_rm_order<<<(unsigned)pf::ceil_div(nbase, RM_THREADS), RM_THREADS, 0, st>>>(
        nbase, start, count, perm, x, y, g, h, sxh, syh, sg);
    PF_TRY(pf::launch_status("k_rm_order"));
    const double qx0 = xb0 / h, qy0 = yb0 / h;
    const double c2 = c * c;
    k_rm_gather<<<(unsigned)pf::ceil_div(ncell, RM_THREADS), RM_THREADS, 0, st>>>(
        nbx, nby, he.ixmin, he.iymin, qx0, qy0, c2, start, count, sxh, syh, sg, acc, flag);
    PF_TRY(pf::launch_status("k_rm_gather"));
    PF_TRY(pf::exclusive_scan_i32(flag, slot, ncell, tmp, total, st));
    k_rm_emit<<<(unsigned)pf::ceil_div(ncell, RM_THREADS), RM_THREADS, 0, st>>>(
        ncell, nby + 3, he.ixmin, he.iymin, h, h05, xb0, yb0, flag, slot, acc, total, capacity,
        x_out, y_out, g_out, ix_out, iy_out);
    PF_TRY(pf::launch_status("k_rm_emit"));
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->host_small, total, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    PF_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t nout = *reinterpret_cast<int32_t *>(ctx->host_small);
    *n_out = nout;
    if (nout > capacity) {
        pf::set_error("pf_remesh: output needs %lld entries, capacity is %lld", (long long)nout,
                      (long long)capacity);
        return PF_ERR_CAPACITY;
    }
    return PF_OK;
}
