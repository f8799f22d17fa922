// remesh.cu -- M4' remesh (pHyFlow Regrid) on a dense lattice window.
//
// Pipeline (all FP64 values, integer cell work bit-exact):
//   1. k_rm_extent : window-left lattice index of every blob,
//        xl = ceil((((x - xb0) - 2h) + 0.5h) / h) - 1     (_regridding.py:157-158)
//      with the same operation order as numpy (IEEE, no FMA contraction:
//      2h and 0.5h are formed on the host); min/max over blobs -> window.
//      [pf_remesh reads the window back: one stream sync.  pf_remesh_window
//       takes the window from the caller instead and never synchronises.]
//   2. k_rm_count  : counting sort of blobs by base cell (xl, yl), base cells
//      ix-major; rank of a blob in its cell from atomicAdd.
//   3. scan of the per-cell counts -> cell starts.
//   4. k_rm_place  : blob index -> its slot.
//   5. k_rm_stencil : one thread per base cell: orders the cell's blobs by
//      input index (every sum below then has a fixed order, independent of
//      atomic timing), then the weights of each of its
//      blobs -- four x weights M4'(ux_a), four y weights M4'(uy_b)
//      (_interpolation_kernels_1d.cpp:75-89; u as _regridding.py:183) or
//      Tutty's -- and the cell's 4 x 4 stencil of partial sums
//      sum over its blobs (in cell order) of (wx_a wy_b) g, stored
//      stencil-major (coalesced).
//   6. k_rm_sum : one thread per output cell (ix, iy): the 16 partial sums of
//      the base cells whose windows cover it, added in fixed (b, a) order;
//      flags cells touched by at least one window (explicit zeros are kept,
//      like the CSR sum of the reference, _regridding.py:200-202).
//   6b. (pf_remesh_population_control only) PopulationControl of the cell
//      values (popctl.cu), which clears the flags of the dropped cells.
//   7. scan of the flags -> output slots, in (ix, iy) order.
//   8. k_rm_emit   : x = ix*h + 0.5h + xb0 (same order as :217-218), g, ix, iy.
// No floating-point atomics: each output value is produced by one thread.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "popctl.cuh"
#include "scan.cuh"
#include "segsort.cuh"

namespace {

constexpr int RM_THREADS = 256;
constexpr int64_t IDX_LIMIT = (int64_t)1 << 30;

struct Extent {
    int32_t ixmin, ixmax, iymin, iymax;
    int32_t bad;  // 1: NaN/Inf coordinate, 2: index outside +-2^30, 4: outside window
    int32_t pad[3];
};

__device__ __forceinline__ int64_t left_index(double x, double b0, double h2, double h05,
                                              double h) {
    // ((x - b0) - 2h) + 0.5h, then / h, ceil, -1 ; each op rounded separately
    const double t = __dadd_rn(__dsub_rn(__dsub_rn(x, b0), h2), h05);
    const double q = __ddiv_rn(t, h);
    return (int64_t)ceil(q) - 1;
}

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

__global__ void __launch_bounds__(RM_THREADS)
k_rm_extent(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double xb0,
            double yb0, double h2, double h05, double h, Extent *e) {
    __shared__ int s_v[5][RM_THREADS / 32];
    int mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN, bad = 0;
    // four independent loads of x and y per thread in flight
    const int64_t stride = (int64_t)gridDim.x * RM_THREADS;
    for (int64_t i0 = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x; i0 < n; i0 += 4 * stride) {
        double xs[4], ys[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = i0 + u * stride;
            xs[u] = i < n ? x[i] : 0.0;
            ys[u] = i < n ? y[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u * stride >= n) continue;
            const double xi = xs[u], yi = ys[u];
            if (!isfinite(xi) || !isfinite(yi)) {
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
    }
    mnx = warp_min(mnx);
    mxx = warp_max(mxx);
    mny = warp_min(mny);
    mxy = warp_max(mxy);
    bad = __reduce_or_sync(0xffffffffu, bad);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_v[0][wid] = mnx;
        s_v[1][wid] = mxx;
        s_v[2][wid] = mny;
        s_v[3][wid] = mxy;
        s_v[4][wid] = bad;
    }
    __syncthreads();
    if (wid == 0) {
        const bool in = lane < RM_THREADS / 32;
        mnx = warp_min(in ? s_v[0][lane] : INT32_MAX);
        mxx = warp_max(in ? s_v[1][lane] : INT32_MIN);
        mny = warp_min(in ? s_v[2][lane] : INT32_MAX);
        mxy = warp_max(in ? s_v[3][lane] : INT32_MIN);
        bad = __reduce_or_sync(0xffffffffu, in ? s_v[4][lane] : 0);
        if (lane == 0) {
            if (mnx != INT32_MAX) {
                atomicMin(&e->ixmin, mnx);
                atomicMax(&e->ixmax, mxx);
                atomicMin(&e->iymin, mny);
                atomicMax(&e->iymax, mxy);
            }
            if (bad) atomicOr(&e->bad, bad);
        }
    }
}

// base cell grid: bx in [0, nbx), by in [0, nby), id = bx*nby + by
__global__ void __launch_bounds__(RM_THREADS)
k_rm_count(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double xb0,
           double yb0, double h2, double h05, double h, int32_t ixmin, int32_t iymin, int64_t nbx,
           int64_t nby, int32_t *__restrict__ cell, int32_t *__restrict__ rank,
           int32_t *__restrict__ count, int32_t *__restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (i >= n) return;
    const double xi = x[i], yi = y[i];
    int64_t a = -1, b = -1;
    if (isfinite(xi) && isfinite(yi)) {
        a = left_index(xi, xb0, h2, h05, h) - ixmin;
        b = left_index(yi, yb0, h2, h05, h) - iymin;
    }
    if (a < 0 || b < 0 || a >= nbx || b >= nby) {  // outside the window: skipped, reported
        cell[i] = -1;
        atomicOr(bad, 4);
        return;
    }
    const int32_t c = (int32_t)(a * nby + b);
    cell[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

__global__ void __launch_bounds__(RM_THREADS)
k_rm_place(int64_t n, const int32_t *__restrict__ cell, const int32_t *__restrict__ rank,
           const int32_t *__restrict__ start, int32_t *__restrict__ perm, int32_t *__restrict__ big,
           int32_t *__restrict__ big_n) {
    const int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (i >= n) return;
    const int32_t c = cell[i];
    if (c < 0) return;
    perm[start[c] + rank[i]] = (int32_t)i;
    // a cell of more than SEG_SMALL blobs (exactly one has this rank) is
    // listed for the segment sort
    if (rank[i] == pf::SEG_SMALL) big[atomicAdd(big_n, 1)] = c;
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

// Tutty redistribution weights (src/python/blobs/base/evolution/_evolution.py:
// 360-404): reference node i = xL + 1 at xi = i h + h/2 + b0, Delta =
// (x - xi)/h, q = 1 - 2 (hNu/h)^2, f = q - Delta^2, g = q - (Delta - 1)^2; the
// four weights of nodes i-1..i+2, each operation rounded as numpy does.
__device__ __forceinline__ void tutty_w(double x, int64_t xl, double h, double h05, double b0,
                                        double q, double (&w)[4]) {
    const double xi = __dadd_rn(__dadd_rn(__dmul_rn((double)(xl + 1), h), h05), b0);
    const double d = __ddiv_rn(__dsub_rn(x, xi), h);
    const double d1 = __dsub_rn(d, 1.0);
    const double f = __dsub_rn(q, __dmul_rn(d, d));
    const double gg = __dsub_rn(q, __dmul_rn(d1, d1));
    const double omd = __dsub_rn(1.0, d);
    w[0] = __dmul_rn(omd, __dmul_rn(0.5, __dsub_rn(__dsub_rn(1.0, f), d)));
    w[1] = __dadd_rn(__dmul_rn(omd, f),
                     __dmul_rn(d, __dmul_rn(0.5, __dsub_rn(__dsub_rn(1.0, gg), d1))));
    w[2] = __dadd_rn(__dmul_rn(omd, __dmul_rn(0.5, __dadd_rn(__dsub_rn(1.0, f), d))),
                     __dmul_rn(d, gg));
    w[3] = __dmul_rn(d, __dmul_rn(0.5, __dadd_rn(__dsub_rn(1.0, gg), d1)));
}

struct W9 {
    double wx[4], wy[4], g;
};

// Order a base cell's blob indices perm[s0 .. s0+cnt) by input index (cells
// hold a few blobs; the atomic ranks of k_rm_count are not reproducible).
__device__ __forceinline__ void sort_cell(int32_t *__restrict__ perm, int s0, int cnt) {
    for (int k = 1; k < cnt; ++k) {
        const int32_t v = perm[s0 + k];
        int j = k - 1;
        while (j >= 0 && perm[s0 + j] > v) {
            perm[s0 + j + 1] = perm[s0 + j];
            --j;
        }
        perm[s0 + j + 1] = v;
    }
}

// The four x weights, four y weights and g of blob i in base cell cc.  M4'
// (TUTTY = false): M4'(ux_a) with the Wee coefficient c^2 = prm; Tutty
// (TUTTY = true): prm = hNu = sqrt(dt nu).
struct WParams {
    double h, xb0, yb0;
    double qx0, qy0;  // xb0/h, yb0/h (IEEE division on the host)
    double prm;       // M4': c^2; Tutty: hNu
};

template <bool TUTTY>
__device__ __forceinline__ W9 blob_w9(int32_t i, int64_t bx, int64_t by, int32_t ixmin,
                                      int32_t iymin, const double *__restrict__ x,
                                      const double *__restrict__ y, const double *__restrict__ g,
                                      const WParams &wp) {
    const double h = wp.h, xb0 = wp.xb0, yb0 = wp.yb0, prm = wp.prm;
    W9 r;
    if (TUTTY) {
        const double rr = __ddiv_rn(prm, h);
        const double q = __dsub_rn(1.0, __dmul_rn(2.0, __dmul_rn(rr, rr)));
        const double h05 = __dmul_rn(0.5, h);
        tutty_w(x[i], ixmin + bx, h, h05, xb0, q, r.wx);
        tutty_w(y[i], iymin + by, h, h05, yb0, q, r.wy);
    } else {
        const double xh = __ddiv_rn(x[i], h), yh = __ddiv_rn(y[i], h);
        const double qx0 = wp.qx0, qy0 = wp.qy0;
        const double ix0 = (double)(ixmin + bx), iy0 = (double)(iymin + by);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            // numpy order: ((ix + 0.5) + xb0/h) - x/h, ix the absolute lattice
            // index (ix0 + a and + 0.5 are exact)
            const double px = __dadd_rn((ix0 + (double)a) + 0.5, qx0);
            const double py = __dadd_rn((iy0 + (double)a) + 0.5, qy0);
            r.wx[a] = m4p(__dsub_rn(px, xh), prm);
            r.wy[a] = m4p(__dsub_rn(py, yh), prm);
        }
    }
    r.g = g[i];
    return r;
}

// Base cell bc = bx*nby + by: the 4 x 4 stencil of partial sums of its blobs,
// part[(a*4 + b) * nbase + bc] = sum over the cell's blobs, in cell order, of
// (wx_a wy_b) g; output cell (bx + a, by + b) of the window grid.  Empty
// cells write zeros (k_rm_sum then loads every entry without waiting for the
// cell's count; adding +0.0 changes no sum).
template <bool TUTTY>
__global__ void __launch_bounds__(RM_THREADS)
k_rm_stencil(int64_t nbase, int64_t nby, int32_t ixmin, int32_t iymin,
             const int32_t *__restrict__ start, const int32_t *__restrict__ count,
             int32_t *__restrict__ perm, const double *__restrict__ x,
             const double *__restrict__ y, const double *__restrict__ g, WParams wp,
             double *__restrict__ part) {
    const int64_t bc = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (bc >= nbase) return;
    const int cnt = count[bc];
    if (cnt > pf::SEG_SMALL) return;  // larger cells: k_rm_stencil_big
    const int s0 = start[bc];
    sort_cell(perm, s0, cnt);  // this thread owns the cell's range
    const int64_t bx = bc / nby, by = bc - bx * nby;
    double p[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) p[k] = 0.0;
    for (int k = 0; k < cnt; ++k) {
        const W9 r = blob_w9<TUTTY>(perm[s0 + k], bx, by, ixmin, iymin, x, y, g, wp);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) p[a * 4 + b] += (r.wx[a] * r.wy[b]) * r.g;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) part[k * nbase + bc] = p[k];
}

// The stencil of each listed cell of more than SEG_SMALL blobs (sorted by
// seg_sort_listed), one CTA per cell: thread t sums the blobs t, t + RM_THREADS,
// ... of the cell (in cell order), then the CTA adds the threads' partial sums
// in a fixed tree order.
template <bool TUTTY>
__global__ void __launch_bounds__(RM_THREADS)
k_rm_stencil_big(const int32_t *__restrict__ list, const int32_t *__restrict__ list_n,
                 int64_t nbase, int64_t nby, int32_t ixmin, int32_t iymin,
                 const int32_t *__restrict__ start, const int32_t *__restrict__ count,
                 const int32_t *__restrict__ perm, const double *__restrict__ x,
                 const double *__restrict__ y, const double *__restrict__ g, WParams wp,
                 double *__restrict__ part) {
    __shared__ double s_p[16][RM_THREADS];
    const int nlist = *list_n;
    for (int k = blockIdx.x; k < nlist; k += gridDim.x) {
        const int64_t bc = list[k];
        const int cnt = count[bc], s0 = start[bc];
        const int64_t bx = bc / nby, by = bc - bx * nby;
        double p[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) p[q] = 0.0;
        for (int j = threadIdx.x; j < cnt; j += RM_THREADS) {
            const W9 r = blob_w9<TUTTY>(perm[s0 + j], bx, by, ixmin, iymin, x, y, g, wp);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) p[a * 4 + b] += (r.wx[a] * r.wy[b]) * r.g;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) s_p[q][threadIdx.x] = p[q];
        __syncthreads();
        for (int w = RM_THREADS / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w)
#pragma unroll
                for (int q = 0; q < 16; ++q) s_p[q][threadIdx.x] += s_p[q][threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x < 16) part[threadIdx.x * nbase + bc] = s_p[threadIdx.x][0];
        __syncthreads();
    }
}

// Output cell grid: ox in [0, nbx+3), oy in [0, nby+3), cid = ox*(nby+3) + oy;
// lattice index ix = ixmin + ox.  Base cell (bx, by) covers ox in bx..bx+3,
// oy in by..by+3.  One thread per output cell adds the stencil entries of its
// covering base cells in fixed (b, a) order.
__global__ void __launch_bounds__(RM_THREADS)
k_rm_sum(int64_t nbx, int64_t nby, const int32_t *__restrict__ count,
         const double *__restrict__ part, double *__restrict__ acc, int32_t *__restrict__ flag) {
    const int64_t noy = nby + 3, ncell = (nbx + 3) * noy;
    const int64_t cid = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (cid >= ncell) return;
    const int64_t ox = cid / noy, oy = cid - ox * noy, nbase = nbx * nby;
    double sum = 0.0;
    int touched = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int64_t by = oy - b;
        if (by < 0 || by >= nby) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int64_t bx = ox - a;
            if (bx < 0 || bx >= nbx) continue;
            const int64_t bc = bx * nby + by;
            touched |= count[bc] != 0;
            sum += part[(a * 4 + b) * nbase + bc];
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

__global__ void k_rm_finish(const int32_t *__restrict__ total, const int32_t *__restrict__ bad,
                            int64_t *__restrict__ n_out_dev, int32_t *__restrict__ status_dev) {
    if (n_out_dev) *n_out_dev = *total;
    if (status_dev) *status_dev = *bad;
}

}  // namespace

namespace pf {

// Dense-window limit: base cells <= max(2^26, 64 n).
static int64_t dense_cell_limit(int64_t n) {
    const int64_t a = (int64_t)1 << 26, b = 64 * n;
    const int64_t lim = a > b ? a : b;
    return lim < ((int64_t)1 << 30) ? lim : ((int64_t)1 << 30);
}

size_t remesh_scratch_bytes(int64_t n, int64_t nbx, int64_t nby) {
    const int64_t nbase = nbx * nby, ncell = (nbx + 3) * (nby + 3);
    const int64_t big = ncell > nbase ? ncell : nbase;
    return align256(4 * n) * 3 + align256(8 * 16 * nbase) + 2 * align256(4 * nbase) +
           align256(4 * (n / (SEG_SMALL + 1) + 3)) +
           align256(8 * ncell) + 2 * align256(4 * ncell) + align256(4 * scan_tmp_ints(big)) +
           3 * align256(16) + align256(sizeof(PcState)) + popctl_scratch_bytes() + 1024;
}

// Everything after the window is known; no host synchronisation.  total_dev
// receives the output count, bad_dev the flags of k_rm_count (4 = a blob
// outside the window, skipped).
pf_status remesh_core(Bump &sc, int64_t n, const double *x, const double *y, const double *g,
                      double h, double xb0, double yb0, double c, int32_t ixmin, int32_t iymin,
                      int64_t nbx, int64_t nby, int64_t capacity, double *xo, double *yo,
                      double *go, int64_t *ixo, int64_t *iyo, int32_t *total, int32_t *bad,
                      cudaStream_t st, const PopCtlArgs *pc, int kernel) {
    const int64_t nbase = nbx * nby, ncell = (nbx + 3) * (nby + 3);
    const int64_t big = ncell > nbase ? ncell : nbase;
    int32_t *cell = (int32_t *)sc.take(4 * n);
    int32_t *rank = (int32_t *)sc.take(4 * n);
    int32_t *perm = (int32_t *)sc.take(4 * n);
    double *part = (double *)sc.take(8 * 16 * nbase);
    // cells listed for the segment sort: [0] count, [1 ..] cell ids
    int32_t *bigc = (int32_t *)sc.take(4 * (n / (SEG_SMALL + 1) + 3));
    int32_t *count = (int32_t *)sc.take(4 * nbase);
    int32_t *start = (int32_t *)sc.take(4 * nbase);
    double *acc = (double *)sc.take(8 * ncell);
    int32_t *flag = (int32_t *)sc.take(4 * ncell);
    int32_t *slot = (int32_t *)sc.take(4 * ncell);
    int32_t *tmp = (int32_t *)sc.take(4 * scan_tmp_ints(big));
    int32_t *nvalid = (int32_t *)sc.take(16);
    if (!nvalid) {
        set_error("remesh: scratch too small");
        return PF_ERR_OOM;
    }
    const double h2 = 2.0 * h, h05 = 0.5 * h;
    const unsigned gn = (unsigned)ceil_div(n, RM_THREADS);
    PF_CUDA_TRY(cudaMemsetAsync(count, 0, 4 * nbase, st));
    k_rm_count<<<gn, RM_THREADS, 0, st>>>(x, y, n, xb0, yb0, h2, h05, h, ixmin, iymin, nbx, nby,
                                          cell, rank, count, bad);
    PF_TRY(launch_status("k_rm_count"));
    PF_TRY(exclusive_scan_i32(count, start, nbase, tmp, nvalid, st));
    PF_CUDA_TRY(cudaMemsetAsync(bigc, 0, sizeof(int32_t), st));
    k_rm_place<<<gn, RM_THREADS, 0, st>>>(n, cell, rank, start, perm, bigc + 1, bigc);
    PF_TRY(launch_status("k_rm_place"));
    // cells above SEG_SMALL blobs (dense clusters); the ranks are free now
    PF_TRY(seg_sort_listed(bigc + 1, bigc, start, count, perm, rank, n / (SEG_SMALL + 1) + 1,
                           st));
    WParams wp{h, xb0, yb0, xb0 / h, yb0 / h, kernel == REMESH_TUTTY ? c : c * c};
    const unsigned gb = (unsigned)ceil_div(nbase, RM_THREADS);
    if (kernel == REMESH_TUTTY)
        k_rm_stencil<true><<<gb, RM_THREADS, 0, st>>>(nbase, nby, ixmin, iymin, start, count, perm,
                                                       x, y, g, wp, part);
    else
        k_rm_stencil<false><<<gb, RM_THREADS, 0, st>>>(nbase, nby, ixmin, iymin, start, count,
                                                        perm, x, y, g, wp, part);
    PF_TRY(launch_status("k_rm_stencil"));
    {
        // a few CTAs suffice (such cells are rare); each loops over the list
        const unsigned gbig = (unsigned)std::min<int64_t>(n / (SEG_SMALL + 1) + 1, 64);
        if (kernel == REMESH_TUTTY)
            k_rm_stencil_big<true><<<gbig, RM_THREADS, 0, st>>>(
                bigc + 1, bigc, nbase, nby, ixmin, iymin, start, count, perm, x, y, g, wp, part);
        else
            k_rm_stencil_big<false><<<gbig, RM_THREADS, 0, st>>>(
                bigc + 1, bigc, nbase, nby, ixmin, iymin, start, count, perm, x, y, g, wp, part);
        PF_TRY(launch_status("k_rm_stencil_big"));
    }
    k_rm_sum<<<(unsigned)ceil_div(ncell, RM_THREADS), RM_THREADS, 0, st>>>(nbx, nby, count, part,
                                                                           acc, flag);
    PF_TRY(launch_status("k_rm_sum"));
    if (pc) {
        PF_TRY(popctl_decide(sc, ncell, acc, flag, *pc, st));
        PF_TRY(popctl_flags(ncell, acc, flag, pc->state, flag, st));
    }
    PF_TRY(exclusive_scan_i32(flag, slot, ncell, tmp, total, st));
    k_rm_emit<<<(unsigned)ceil_div(ncell, RM_THREADS), RM_THREADS, 0, st>>>(
        ncell, nby + 3, ixmin, iymin, h, h05, xb0, yb0, flag, slot, acc, total, capacity, xo, yo,
        go, ixo, iyo);
    return launch_status("k_rm_emit");
}

}  // namespace pf

namespace {

// pf_remesh and pf_remesh_population_control: window from the blobs (one
// synchronisation), remesh, optional population control of the cells
// (popctl = {gThresholdLocal, gThresholdGlobal}), output count read back.
pf_status remesh_sync(pf_ctx *ctx, int64_t n, const double *x, const double *y, const double *g,
                      double h, double xb0, double yb0, double c, int64_t capacity,
                      double *x_out, double *y_out, double *g_out, int64_t *ix_out,
                      int64_t *iy_out, int64_t *n_out, const double *popctl, double *thr_used,
                      int kernel, void *stream) {
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
    PF_TRY(pf::arena_reserve(ctx, 4096));
    Extent *ext = static_cast<Extent *>(pf::arena_take(ctx, sizeof(Extent)));
    k_rm_extent_init<<<1, 1, 0, st>>>(ext);
    PF_TRY(pf::launch_status("k_rm_extent_init"));
    {
        int64_t grid = pf::ceil_div(n, RM_THREADS);
        const int64_t cap = (int64_t)ctx->num_sms * 8;
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
    if (nbx * nby > pf::dense_cell_limit(n) || (nbx + 3) * (nby + 3) >= ((int64_t)1 << 31)) {
        pf::set_error("pf_remesh: lattice window %lld x %lld is too large for %lld blobs",
                      (long long)nbx, (long long)nby, (long long)n);
        return PF_ERR_INVALID_ARG;
    }
    PF_TRY(pf::arena_reserve(ctx, pf::remesh_scratch_bytes(n, nbx, nby)));
    pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
    int32_t *total = (int32_t *)sc.take(16);
    int32_t *bad = (int32_t *)sc.take(16);
    pf::PcState *state = (pf::PcState *)sc.take(sizeof(pf::PcState));
    PF_CUDA_TRY(cudaMemsetAsync(bad, 0, 4, st));
    pf::PopCtlArgs pc{popctl ? popctl[0] : 0.0, popctl ? popctl[1] : 0.0, state};
    PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, he.ixmin, he.iymin, nbx, nby, capacity,
                           x_out, y_out, g_out, ix_out, iy_out, total, bad, st,
                           popctl ? &pc : nullptr, kernel));
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->host_small, total, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    if (popctl)
        PF_CUDA_TRY(cudaMemcpyAsync(ctx->host_small + 1, &state->thr, sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
    PF_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t nout = *reinterpret_cast<int32_t *>(ctx->host_small);
    *n_out = nout;
    if (popctl && thr_used) memcpy(thr_used, ctx->host_small + 1, sizeof(double));
    if (nout > capacity) {
        pf::set_error("pf_remesh: output needs %lld entries, capacity is %lld", (long long)nout,
                      (long long)capacity);
        return PF_ERR_CAPACITY;
    }
    return PF_OK;
}

}  // namespace

extern "C" pf_status pf_remesh(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                               const double *g, double h, double xb0, double yb0, double c,
                               int64_t capacity, double *x_out, double *y_out, double *g_out,
                               int64_t *ix_out, int64_t *iy_out, int64_t *n_out, void *stream) {
    pf::clear_error();
    return remesh_sync(ctx, n, x, y, g, h, xb0, yb0, c, capacity, x_out, y_out, g_out, ix_out,
                       iy_out, n_out, nullptr, nullptr, pf::REMESH_M4, stream);
}

extern "C" pf_status pf_remesh_tutty(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                     const double *g, double h, double xb0, double yb0,
                                     double hnu, int64_t capacity, double *x_out, double *y_out,
                                     double *g_out, int64_t *ix_out, int64_t *iy_out,
                                     int64_t *n_out, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(std::isfinite(hnu) && hnu >= 0.0, "pf_remesh_tutty: hnu must be >= 0 and finite");
    return remesh_sync(ctx, n, x, y, g, h, xb0, yb0, hnu, capacity, x_out, y_out, g_out, ix_out,
                       iy_out, n_out, nullptr, nullptr, pf::REMESH_TUTTY, stream);
}

extern "C" pf_status pf_remesh_population_control(
    pf_ctx *ctx, int64_t n, const double *x, const double *y, const double *g, double h,
    double xb0, double yb0, double c, double g_threshold_local, double g_threshold_global,
    int64_t capacity, double *x_out, double *y_out, double *g_out, int64_t *ix_out,
    int64_t *iy_out, int64_t *n_out, double *threshold_used, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(n_out != nullptr, "pf_remesh_population_control: n_out is NULL");
    *n_out = 0;
    PF_TRY(pf::popctl_check(g_threshold_local, g_threshold_global,
                            "pf_remesh_population_control"));
    const double pc[2] = {g_threshold_local, g_threshold_global};
    if (threshold_used) *threshold_used = g_threshold_local;
    return remesh_sync(ctx, n, x, y, g, h, xb0, yb0, c, capacity, x_out, y_out, g_out, ix_out,
                       iy_out, n_out, pc, threshold_used, pf::REMESH_M4, stream);
}

extern "C" pf_status pf_remesh_window(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                      const double *g, double h, double xb0, double yb0, double c,
                                      int64_t ixmin, int64_t iymin, int64_t nbx, int64_t nby,
                                      int64_t capacity, double *x_out, double *y_out,
                                      double *g_out, int64_t *ix_out, int64_t *iy_out,
                                      int64_t *n_out_dev, int32_t *status_dev, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_remesh_window: NULL context");
    PF_CHECK_ARG(n >= 0 && n < ((int64_t)1 << 31), "pf_remesh_window: bad n");
    PF_CHECK_ARG(std::isfinite(h) && h > 0.0, "pf_remesh_window: bad h");
    PF_CHECK_ARG(std::isfinite(xb0) && std::isfinite(yb0) && std::isfinite(c),
                 "pf_remesh_window: bounds and c must be finite");
    PF_CHECK_ARG(nbx > 0 && nby > 0 && (nbx + 3) * (nby + 3) < ((int64_t)1 << 31),
                 "pf_remesh_window: bad window %lld x %lld", (long long)nbx, (long long)nby);
    PF_CHECK_ARG(ixmin > -((int64_t)1 << 30) && iymin > -((int64_t)1 << 30) &&
                     ixmin + nbx < ((int64_t)1 << 30) && iymin + nby < ((int64_t)1 << 30),
                 "pf_remesh_window: window outside +-2^30");
    PF_CHECK_ARG(n == 0 || (x && y && g), "pf_remesh_window: NULL input array");
    PF_CHECK_ARG(capacity >= 0 && (capacity == 0 || (x_out && y_out && g_out)),
                 "pf_remesh_window: bad output arrays");
    PF_CHECK_ARG(n_out_dev != nullptr, "pf_remesh_window: n_out_dev is NULL");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PF_TRY(pf::arena_reserve(ctx, pf::remesh_scratch_bytes(n, nbx, nby)));
    pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
    int32_t *total = (int32_t *)sc.take(16);
    int32_t *bad = (int32_t *)sc.take(16);
    PF_CUDA_TRY(cudaMemsetAsync(total, 0, 4, st));
    PF_CUDA_TRY(cudaMemsetAsync(bad, 0, 4, st));
    if (n > 0)
        PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, (int32_t)ixmin, (int32_t)iymin, nbx,
                               nby, capacity, x_out, y_out, g_out, ix_out, iy_out, total, bad, st));
    k_rm_finish<<<1, 1, 0, st>>>(total, bad, n_out_dev, status_dev);
    return pf::launch_status("k_rm_finish");
}
