// remesh.cu -- M4' remesh (pHyFlow Regrid) on a dense lattice window.
//
// Pipeline (all FP64 values, integer cell work bit-exact), ten stream-ordered
// steps with no host synchronisation:
//   0. one memset: the call's RmHead and the base-cell counts.
//   1. k_rm_extent : window-left lattice index of every blob,
//        xl = ceil((((x - xb0) - 2h) + 0.5h) / h) - 1     (_regridding.py:157-158)
//      with the same operation order as numpy (IEEE, no FMA contraction:
//      2h and 0.5h are formed on the host); min/max over blobs; the last CTA
//      to finish turns the extent into the window and checks it against the
//      scratch capacity.  [k_rm_set_window instead when the caller gives the
//      window.]
//   2. k_rm_count  : counting sort of blobs by base cell (xl, yl), base cells
//      ix-major; rank of a blob in its cell from atomicAdd.
//   3. k_rm_scan_up / k_rm_scan_down : two exclusive scans in the same two
//      launches -- base-cell counts -> cell starts, and the touched flags of
//      the output cells -> output slots in (ix, iy) order.  An output cell is
//      touched when one of the 4 x 4 base cells whose windows cover it holds a
//      blob (explicit zeros are kept, like the CSR sum of the reference,
//      _regridding.py:200-202), so the output order is known before any value.
//   4. k_rm_place  : blob -> its slot in cell order: a 32-byte record {x/h,
//      y/h, g, index} (the IEEE quotients of _regridding.py:183 computed once
//      per blob; x, y for Tutty).
//   5. seg_sort_listed + k_rm_stencil_big : cells of more than SEG_SMALL blobs
//      (dense clusters), one CTA per cell, stencil partial sums to a side table.
//   6. k_rm_tile   : one CTA per tile of 8 x 29 output cells.  Each thread
//      takes one of the 11 x 32 base cells feeding the tile (a warp per base
//      row), walks the cell's blobs in input-index order (found in
//      registers), forms their four x weights M4'(ux_a) and four y weights
//      M4'(uy_b) (_interpolation_kernels_1d.cpp:75-89; with c = 0 each node on
//      its known branch, m4p_outer / m4p_inner) or Tutty's, and
//      accumulates the cell's 4 x 4 stencil of partial sums sum (wx_a wy_b) g
//      in shared memory.  Then each output cell adds the 16 partial sums of the base
//      cells that cover it in fixed (b, a) order and writes x = ix*h + 0.5h +
//      xb0 (same order as :217-218), g, ix, iy at its slot.
//      [pf_remesh_population_control: the cell values and flags go to HBM
//       instead, PopulationControl (popctl.cu) clears the flags of the dropped
//       cells, then a scan and k_rm_emit.]
//   7. k_rm_finish : output count and status words.
// No floating-point atomics: each partial and each output value is produced
// by one thread in a fixed order, so results are bitwise reproducible.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "remesh.cuh"
#include "scan.cuh"
#include "segsort.cuh"

namespace {

using pf::RM_IDX_OFF;
using pf::RmHead;

constexpr int RM_THREADS = 256;
constexpr int32_t IDX_LIMIT = 1 << 30;

// scan tiles
constexpr int SC_THREADS = 512;
constexpr int SC_ITEMS = 8;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

// output tile of k_rm_tile: TOX rows (ix) x TOY columns (iy) of output cells,
// fed by TBX x TBY base cells (TBY = 32: one warp per base row)
constexpr int TOX = 8, TOY = 29;
constexpr int TBX = TOX + 3, TBY = TOY + 3;
constexpr int TILE_THREADS = TBX * TBY;  // 352
constexpr int TILE_PREF = 4;  // cell sizes whose blob order is found in registers
static_assert(TBY == 32, "one warp per base row");

struct Win {
    int64_t ixmin, iymin, nbx, nby, nbase, nox, noy, ncell;
    const int32_t *rows, *cols;  // compressed window (else null)
};

__device__ __forceinline__ bool load_win(const RmHead *hd, Win &w) {
    if (!hd->ok) return false;
    w.ixmin = hd->ixmin;
    w.iymin = hd->iymin;
    w.nbx = hd->nbx;
    w.nby = hd->nby;
    w.nbase = w.nbx * w.nby;
    w.nox = w.nbx + 3;
    w.noy = w.nby + 3;
    w.ncell = w.nox * w.noy;
    w.rows = hd->rows;
    w.cols = hd->cols;
    return true;
}

// Lattice row / column of window row bx / column by.  In a compressed window
// the rows after an occupied base row bx are rows[bx] + 1 .. + 3 (they are in
// the list by construction), so stencil neighbours stay window neighbours.
__device__ __forceinline__ int64_t lat_x(const Win &w, int64_t bx) {
    if (!w.rows) return w.ixmin + bx;
    // past the list (only the empty border rows of the window): extrapolated
    return bx < w.nbx ? (int64_t)w.rows[bx] : (int64_t)w.rows[w.nbx - 1] + (bx - (w.nbx - 1));
}
__device__ __forceinline__ int64_t lat_y(const Win &w, int64_t by) {
    if (!w.cols) return w.iymin + by;
    return by < w.nby ? (int64_t)w.cols[by] : (int64_t)w.cols[w.nby - 1] + (by - (w.nby - 1));
}

// Window index of lattice index v in the sorted list a[0 .. n), -1 if absent.
__device__ __forceinline__ int64_t find_sorted(const int32_t *__restrict__ a, int64_t n,
                                               int64_t v) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < n && (int64_t)a[lo] == v) ? lo : -1;
}

// One blob in cell order, written by k_rm_place as one whole 32-byte sector:
// v1, v2 = x/h, y/h (M4': the IEEE quotients of the reference's u = (ix +
// 0.5 + xb0/h) - x/h) or x, y (Tutty), its circulation and input index.
// (Weights computed here instead, 64 more bytes per blob, measured slower:
// k_rm_place 26 -> 60 us, k_rm_tile 94 -> 78 us at N = 2^20.)
struct WRec {
    double v1, v2, g;
    long long idx;
};
static_assert(sizeof(WRec) == 32, "WRec layout");

// One 32-byte record written by a single 256-bit store (sm_100), so the
// sector is written whole.
__device__ __forceinline__ void st_rec(WRec *r, double a, double b, double c, double d) {
    asm volatile("st.global.v4.b64 [%0], {%1, %2, %3, %4};" ::"l"(r), "d"(a), "d"(b), "d"(c),
                 "d"(d)
                 : "memory");
}

__device__ __forceinline__ int64_t left_index(double x, double b0, double h2, double h05,
                                              double h) {
    // ((x - b0) - 2h) + 0.5h, then / h, ceil, -1 ; each op rounded separately
    const double t = __dadd_rn(__dsub_rn(__dsub_rn(x, b0), h2), h05);
    const double q = __ddiv_rn(t, h);
    return (int64_t)ceil(q) - 1;
}

__device__ __forceinline__ int warp_max(int v) {
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum of four FP64 values in a fixed order (warp butterflies, then
// warp 0 over the warps' sums); the result is valid in thread 0.
template <int THREADS>
__device__ __forceinline__ void block_sum4(double (&m)[4], double (*s_w)[4]) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o; o >>= 1) m[q] += __shfl_xor_sync(0xffffffffu, m[q], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) s_w[wid][q] = m[q];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 1; k < (THREADS + 31) / 32; ++k)
#pragma unroll
            for (int q = 0; q < 4; ++q) m[q] += s_w[k][q];
}

// Grid-wide moments: every CTA's block sum goes to part[4 blockIdx ..]; the
// last CTA to finish (ticket) adds the CTAs' sums in a fixed order (thread t
// takes CTAs t, t + THREADS, ...; then block_sum4) into out[0..4).  Every
// thread of every CTA must call it (no early return before).
template <int THREADS>
__device__ __forceinline__ void grid_moments(double (&m)[4], double *__restrict__ part,
                                             unsigned *ticket, double *out) {
    __shared__ double s_w[(THREADS + 31) / 32][4];
    __shared__ int s_last;
    block_sum4<THREADS>(m, s_w);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) part[4 * (int64_t)blockIdx.x + q] = m[q];
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
#pragma unroll
    for (int q = 0; q < 4; ++q) m[q] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += THREADS)
#pragma unroll
        for (int q = 0; q < 4; ++q) m[q] += __ldcg(&part[4 * (int64_t)b + q]);
    block_sum4<THREADS>(m, s_w);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = m[q];
}

__device__ __forceinline__ void add_moments(double (&m)[4], double x, double y, double g) {
    m[0] += g;
    m[1] += g * x;
    m[2] += g * y;
    m[3] += fabs(g);
}

// Window extent from the blobs; the last CTA to finish sets the window.
__global__ void __launch_bounds__(RM_THREADS)
k_rm_extent(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double xb0,
            double yb0, double h2, double h05, double h, RmHead *hd, int64_t cap_base,
            int64_t cap_cell, int64_t limit, int32_t *__restrict__ xl_out,
            int32_t *__restrict__ yl_out) {
    __shared__ int s_v[5][RM_THREADS / 32];
    __shared__ int s_last;
    int xhi = 0, xlo = 0, yhi = 0, ylo = 0, bad = 0;
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
            const int64_t iu = i0 + u * stride;
            if (!isfinite(xi) || !isfinite(yi)) {
                bad |= 1;
                xl_out[iu] = yl_out[iu] = INT32_MIN;
                continue;
            }
            const int64_t a = left_index(xi, xb0, h2, h05, h);
            const int64_t b = left_index(yi, yb0, h2, h05, h);
            if (a <= -IDX_LIMIT || a >= IDX_LIMIT || b <= -IDX_LIMIT || b >= IDX_LIMIT) {
                bad |= 2;
                xl_out[iu] = yl_out[iu] = INT32_MIN;
                continue;
            }
            // for k_rm_count (|a|, |b| < 2^30 here)
            xl_out[iu] = (int32_t)a;
            yl_out[iu] = (int32_t)b;
            xhi = max(xhi, (int)a + RM_IDX_OFF);
            xlo = max(xlo, RM_IDX_OFF - (int)a);
            yhi = max(yhi, (int)b + RM_IDX_OFF);
            ylo = max(ylo, RM_IDX_OFF - (int)b);
        }
    }
    xhi = warp_max(xhi);
    xlo = warp_max(xlo);
    yhi = warp_max(yhi);
    ylo = warp_max(ylo);
    bad = __reduce_or_sync(0xffffffffu, bad);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_v[0][wid] = xhi;
        s_v[1][wid] = xlo;
        s_v[2][wid] = yhi;
        s_v[3][wid] = ylo;
        s_v[4][wid] = bad;
    }
    __syncthreads();
    if (wid == 0) {
        const bool in = lane < RM_THREADS / 32;
        xhi = warp_max(in ? s_v[0][lane] : 0);
        xlo = warp_max(in ? s_v[1][lane] : 0);
        yhi = warp_max(in ? s_v[2][lane] : 0);
        ylo = warp_max(in ? s_v[3][lane] : 0);
        bad = __reduce_or_sync(0xffffffffu, in ? s_v[4][lane] : 0);
        if (lane == 0) {
            if (xhi) {
                atomicMax(&hd->xhi, xhi);
                atomicMax(&hd->xlo, xlo);
                atomicMax(&hd->yhi, yhi);
                atomicMax(&hd->ylo, ylo);
            }
            if (bad) atomicOr(&hd->bad, bad);
            __threadfence();
            s_last = atomicAdd(&hd->ticket, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    // every other CTA's updates are visible (fence before its ticket)
    __threadfence();
    const int32_t b = atomicOr(&hd->bad, 0);
    const int32_t X1 = atomicMax(&hd->xhi, 0), X0 = atomicMax(&hd->xlo, 0);
    const int32_t Y1 = atomicMax(&hd->yhi, 0), Y0 = atomicMax(&hd->ylo, 0);
    int ok = 0;
    int64_t ixmin = 0, iymin = 0, nbx = 0, nby = 0, ncell = 0;
    if (!(b & 3) && X1 > 0 && Y1 > 0) {
        ixmin = (int64_t)RM_IDX_OFF - X0;
        iymin = (int64_t)RM_IDX_OFF - Y0;
        nbx = ((int64_t)X1 - RM_IDX_OFF) - ixmin + 1;
        nby = ((int64_t)Y1 - RM_IDX_OFF) - iymin + 1;
        const int64_t nbase = nbx * nby;
        ncell = (nbx + 3) * (nby + 3);
        ok = nbase <= cap_base && nbase <= limit && ncell <= cap_cell &&
             ncell < ((int64_t)1 << 31);
        if (!ok) atomicOr(&hd->bad, 8);
    }
    hd->ixmin = (int32_t)ixmin;
    hd->iymin = (int32_t)iymin;
    hd->nbx = (int32_t)nbx;
    hd->nby = (int32_t)nby;
    hd->ncell = ok ? ncell : 0;
    hd->ok = ok;
}

__global__ void k_rm_set_window(RmHead *hd, int32_t ixmin, int32_t iymin, int32_t nbx,
                                int32_t nby, const int32_t *rows, const int32_t *cols) {
    hd->rows = rows;
    hd->cols = cols;
    hd->ixmin = ixmin;
    hd->iymin = iymin;
    hd->nbx = nbx;
    hd->nby = nby;
    hd->ncell = ((int64_t)nbx + 3) * ((int64_t)nby + 3);
    hd->ok = 1;
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

// The four x weights and four y weights of a blob at (xv, yv) in the base cell
// with absolute lattice indices (ix0, iy0).  M4' (TUTTY = false): M4'(ux_a)
// with the Wee coefficient c^2 = prm; Tutty (TUTTY = true): prm = hNu.
struct WParams {
    double h, h05, xb0, yb0;
    double qx0, qy0;  // xb0/h, yb0/h (IEEE division on the host)
    double prm;       // M4': c^2; Tutty: hNu
};

template <bool TUTTY>
__device__ __forceinline__ void blob_w8(double xv, double yv, int64_t ix0, int64_t iy0,
                                        const WParams &wp, double (&wx)[4], double (&wy)[4]) {
    const double h = wp.h, prm = wp.prm;
    if (TUTTY) {
        const double rr = __ddiv_rn(prm, h);
        const double q = __dsub_rn(1.0, __dmul_rn(2.0, __dmul_rn(rr, rr)));
        tutty_w(xv, ix0, h, wp.h05, wp.xb0, q, wx);
        tutty_w(yv, iy0, h, wp.h05, wp.yb0, q, wy);
    } else {
        const double xh = __ddiv_rn(xv, h), yh = __ddiv_rn(yv, h);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            // numpy order: ((ix + 0.5) + xb0/h) - x/h, ix the absolute lattice
            // index (ix0 + a and + 0.5 are exact)
            const double px = __dadd_rn(((double)ix0 + (double)a) + 0.5, wp.qx0);
            const double py = __dadd_rn(((double)iy0 + (double)a) + 0.5, wp.qy0);
            wx[a] = m4p(__dsub_rn(px, xh), prm);
            wy[a] = m4p(__dsub_rn(py, yh), prm);
        }
    }
}

// base cell grid: bx in [0, nbx), by in [0, nby), id = bx*nby + by
__global__ void __launch_bounds__(RM_THREADS)
k_rm_count(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double xb0,
           double yb0, double h2, double h05, double h, RmHead *hd, int32_t *__restrict__ cell,
           int32_t *__restrict__ rank, int32_t *__restrict__ count, bool pre) {
    Win w;
    if (!load_win(hd, w)) return;
    const int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (i >= n) return;
    int64_t a = -1, b = -1;
    if (pre) {  // left indices from k_rm_extent, in cell[] / rank[] (INT32_MIN: not finite)
        const int32_t pa = cell[i], pb = rank[i];
        if (pa != INT32_MIN) {
            a = pa - w.ixmin;
            b = pb - w.iymin;
        }
    } else if (isfinite(x[i]) && isfinite(y[i])) {
        const double xi = x[i], yi = y[i];
        a = left_index(xi, xb0, h2, h05, h);
        b = left_index(yi, yb0, h2, h05, h);
        a = w.rows ? find_sorted(w.rows, w.nbx, a) : a - w.ixmin;
        b = w.cols ? find_sorted(w.cols, w.nby, b) : b - w.iymin;
    }
    if (a < 0 || b < 0 || a >= w.nbx || b >= w.nby) {  // outside the window: skipped, reported
        cell[i] = -1;
        atomicOr(&hd->bad, 4);
        return;
    }
    const int32_t c = (int32_t)(a * w.nby + b);
    if (!PF_IDX_OK(c, (int64_t)w.nbx * w.nby, 101)) {
        cell[i] = -1;
        return;
    }
    cell[i] = c;
    rank[i] = atomicAdd(&count[c], 1);
}

// Lattice left indices of every blob (for the compressed window of a sparse
// blob set; the coordinates are finite and in range: checked before).
__global__ void __launch_bounds__(RM_THREADS)
k_rm_left_indices(const double *__restrict__ x, const double *__restrict__ y, int64_t n,
                  double xb0, double yb0, double h2, double h05, double h,
                  int32_t *__restrict__ xl, int32_t *__restrict__ yl) {
    const int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (i >= n) return;
    xl[i] = (int32_t)left_index(x[i], xb0, h2, h05, h);
    yl[i] = (int32_t)left_index(y[i], yb0, h2, h05, h);
}

// OR over a in [0, 4) of "base cell (ox - a, by) of the window holds a blob"
__device__ __forceinline__ int col_or(const int32_t *__restrict__ count, const Win &w, int64_t ox,
                                      int64_t by) {
    if (by < 0 || by >= w.nby) return 0;
    int f = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int64_t bx = ox - a;
        if (bx >= 0 && bx < w.nbx) f |= count[bx * w.nby + by] != 0;
    }
    return f;
}

// The SC_ITEMS values of thread `base` of scan part 0 (base-cell counts) or
// part 1 (touched flags of output cells: a base cell (ox - a, oy - b), a, b in
// [0, 4), of the window holds a blob; the column ORs roll along oy).
__device__ __forceinline__ void scan_items(int part, const int32_t *__restrict__ count,
                                           const Win &w, int64_t base, int (&v)[SC_ITEMS]) {
    if (part == 0) {
#pragma unroll
        for (int k = 0; k < SC_ITEMS; ++k) v[k] = base + k < w.nbase ? count[base + k] : 0;
    } else {
        int64_t ox = base / w.noy, oy = base - ox * w.noy;
        int c1 = col_or(count, w, ox, oy - 1), c2 = col_or(count, w, ox, oy - 2),
            c3 = col_or(count, w, ox, oy - 3);
#pragma unroll
        for (int k = 0; k < SC_ITEMS; ++k) {
            const int c0 = col_or(count, w, ox, oy);
            v[k] = base + k < w.ncell ? (c0 | c1 | c2 | c3) : 0;
            c3 = c2;
            c2 = c1;
            c1 = c0;
            if (++oy == w.noy) {  // next output row: its columns -1..-3 are empty
                oy = 0;
                ++ox;
                c1 = c2 = c3 = 0;
            }
        }
    }
}

__device__ __forceinline__ int block_sum(int v, int *s_w) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = __reduce_add_sync(0xffffffffu, v);
    __syncthreads();
    if (lane == 0) s_w[wid] = v;
    __syncthreads();
    int t = 0;
#pragma unroll
    for (int k = 0; k < SC_THREADS / 32; ++k) t += s_w[k];
    return t;
}

// Tile sums of both scans (grid: capacity tiles of part 0, then of part 1).
__global__ void __launch_bounds__(SC_THREADS)
k_rm_scan_up(const RmHead *__restrict__ hd, const int32_t *__restrict__ count, int64_t ntA_cap,
             int32_t *__restrict__ tsA, int32_t *__restrict__ tsB, uint8_t *__restrict__ oflag) {
    __shared__ int s_w[SC_THREADS / 32];
    Win w;
    if (!load_win(hd, w)) return;
    const int part = (int64_t)blockIdx.x < ntA_cap ? 0 : 1;
    const int64_t t = part ? (int64_t)blockIdx.x - ntA_cap : (int64_t)blockIdx.x;
    const int64_t len = part ? w.ncell : w.nbase;
    if (t * SC_TILE >= len) return;
    const int64_t base = t * SC_TILE + (int64_t)threadIdx.x * SC_ITEMS;
    int v[SC_ITEMS];
    scan_items(part, count, w, base, v);
    if (part == 1 && base < len) {  // the flags, for k_rm_scan_down (8 bytes, aligned)
        unsigned long long packed = 0;
#pragma unroll
        for (int k = 0; k < SC_ITEMS; ++k) packed |= (unsigned long long)(v[k] & 1) << (8 * k);
        *reinterpret_cast<unsigned long long *>(oflag + base) = packed;
    }
    int s = 0;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) s += v[k];
    s = block_sum(s, s_w);
    if (threadIdx.x == 0) (part ? tsB : tsA)[t] = s;
}

// Exclusive scans: the tile's offset is the sum of the earlier tiles' sums
// (added up by the CTA itself), then a block scan of the tile.  Part 1's
// last tile writes the output count.
__global__ void __launch_bounds__(SC_THREADS)
k_rm_scan_down(RmHead *__restrict__ hd, const int32_t *__restrict__ count, int64_t ntA_cap,
               const int32_t *__restrict__ tsA, const int32_t *__restrict__ tsB,
               const uint8_t *__restrict__ oflag, int32_t *__restrict__ start,
               int32_t *__restrict__ slot) {
    __shared__ int s_w[SC_THREADS / 32];
    __shared__ int s_x[SC_THREADS / 32 + 1];
    Win w;
    if (!load_win(hd, w)) return;
    const int part = (int64_t)blockIdx.x < ntA_cap ? 0 : 1;
    const int64_t t = part ? (int64_t)blockIdx.x - ntA_cap : (int64_t)blockIdx.x;
    const int64_t len = part ? w.ncell : w.nbase;
    if (t * SC_TILE >= len) return;
    const int32_t *ts = part ? tsB : tsA;
    int32_t *out = part ? slot : start;
    int pre = 0;
    for (int64_t j = threadIdx.x; j < t; j += SC_THREADS) pre += ts[j];
    pre = block_sum(pre, s_w);
    const int64_t base = t * SC_TILE + (int64_t)threadIdx.x * SC_ITEMS;
    int v[SC_ITEMS];
    if (part == 0) {
        scan_items(0, count, w, base, v);
    } else {
        const unsigned long long packed =
            base < len ? *reinterpret_cast<const unsigned long long *>(oflag + base) : 0ull;
#pragma unroll
        for (int k = 0; k < SC_ITEMS; ++k) v[k] = (int)((packed >> (8 * k)) & 1ull);
    }
    int s = 0;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) s += v[k];
    // block exclusive scan of the thread sums
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) s_x[wid] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < SC_THREADS / 32; ++k) {
            const int q = s_x[k];
            s_x[k] = acc;
            acc += q;
        }
        s_x[SC_THREADS / 32] = acc;
    }
    __syncthreads();
    int ex = pre + s_x[wid] + inc - s;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; ++k) {
        if (base + k < len) out[base + k] = ex;
        ex += v[k];
    }
    if (part == 1 && threadIdx.x == 0 && (t + 1) * SC_TILE >= len)
        hd->total = pre + s_x[SC_THREADS / 32];
}

// Blob -> its slot in cell order: a 32-byte record (x/h and y/h -- the
// divisions done once per blob, with every thread busy -- or x, y for Tutty,
// g, its index); and the FP64 moments of the blobs placed.
template <bool TUTTY>
__global__ void __launch_bounds__(RM_THREADS)
k_rm_place(int64_t n, RmHead *hd, const int32_t *__restrict__ cell,
           const int32_t *__restrict__ rank, const int32_t *__restrict__ start,
           const double *__restrict__ x, const double *__restrict__ y,
           const double *__restrict__ g, WParams wp, WRec *__restrict__ recs,
           int32_t *__restrict__ big, double *__restrict__ mpart) {
    Win w;
    if (!load_win(hd, w)) return;  // the same for every CTA
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    // grid-stride: a few blobs per thread, one moment reduction per CTA
    for (int64_t i = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * RM_THREADS) {
        const int32_t c = cell[i];
        if (c < 0) continue;
        const int32_t r = rank[i];
        const int64_t p = (int64_t)start[c] + r;
        if (!PF_IDX_OK(p, n, 102)) continue;
        const double xi = x[i], yi = y[i], gi = g[i];
        const double v1 = TUTTY ? xi : __ddiv_rn(xi, wp.h);
        const double v2 = TUTTY ? yi : __ddiv_rn(yi, wp.h);
        // the whole 32-byte sector in one store (records are 32-byte aligned)
        st_rec(recs + p, v1, v2, gi, __longlong_as_double((long long)i));
        add_moments(m, xi, yi, gi);
        // a cell of more than SEG_SMALL blobs (exactly one has this rank) is
        // listed for the segment sort
        if (r == pf::SEG_SMALL) big[atomicAdd(&hd->big_n, 1)] = c;
    }
    grid_moments<RM_THREADS>(m, mpart, &hd->ticket_in, hd->mom);
}

// The input indices of each listed cell of more than SEG_SMALL blobs, from its
// records into vals[start ..] (for the segment sort).
__global__ void __launch_bounds__(RM_THREADS)
k_rm_big_gather(const int32_t *__restrict__ list, const RmHead *__restrict__ hd,
                const int32_t *__restrict__ start, const int32_t *__restrict__ count,
                const WRec *__restrict__ recs, int32_t *__restrict__ vals) {
    if (!hd->ok) return;
    const int nlist = hd->big_n;
    for (int k = blockIdx.x; k < nlist; k += gridDim.x) {
        const int64_t bc = list[k];
        const int cnt = count[bc], s0 = start[bc];
        for (int j = threadIdx.x; j < cnt; j += RM_THREADS) vals[s0 + j] = (int32_t)recs[s0 + j].idx;
    }
}

// Weights of the tile kernel: M4' with any c, M4' with c = 0, Tutty.
constexpr int WK_M4 = 0, WK_M4_PLAIN = 1, WK_TUTTY = 2;

// M4' at c = 0 on the node's known branch.  x_L = ceil(s) - 1 with s = x/h -
// xb0/h - 1.5 (_regridding.py:162) puts u_a = x_L + a - (s + 1) in [-2, -1),
// [-1, 0), [0, 1), [1, 2) for a = 0..3, so nodes 0 and 3 take the outer
// polynomial and nodes 1 and 2 the inner one.  At |u| = 1 both are 0 (which is
// also the reference's value there), and where rounding puts a computed u an
// ulp across 1 both polynomials are within an ulp-sized amount of 0, so the
// weights match the value-branched m4p to ~1e-16 absolute.
__device__ __forceinline__ double m4p_outer(double u) {
    const double a = fabs(u);
    const double t = 2.0 - a;
    return 0.5 * (t * t) * (1.0 - a);
}
__device__ __forceinline__ double m4p_inner(double u) {
    const double a = fabs(u);
    const double a2 = u * u;
    return 1.0 - 2.5 * a2 + 1.5 * (a2 * a);
}

// blob_w8 from a record's values: M4' takes x/h, y/h as computed in
// k_rm_place (the same IEEE quotients blob_w8 forms), Tutty takes x, y.
template <int WK>
__device__ __forceinline__ void rec_w8(double v1, double v2, int64_t ix0, int64_t iy0,
                                       const WParams &wp, double (&wx)[4], double (&wy)[4]) {
    if (WK == WK_TUTTY) {
        blob_w8<true>(v1, v2, ix0, iy0, wp, wx, wy);
    } else if (WK == WK_M4_PLAIN) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double ux = __dsub_rn(__dadd_rn(((double)ix0 + (double)a) + 0.5, wp.qx0), v1);
            const double uy = __dsub_rn(__dadd_rn(((double)iy0 + (double)a) + 0.5, wp.qy0), v2);
            wx[a] = (a == 0 || a == 3) ? m4p_outer(ux) : m4p_inner(ux);
            wy[a] = (a == 0 || a == 3) ? m4p_outer(uy) : m4p_inner(uy);
        }
    } else {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double px = __dadd_rn(((double)ix0 + (double)a) + 0.5, wp.qx0);
            const double py = __dadd_rn(((double)iy0 + (double)a) + 0.5, wp.qy0);
            wx[a] = m4p(__dsub_rn(px, v1), wp.prm);
            wy[a] = m4p(__dsub_rn(py, v2), wp.prm);
        }
    }
}

// The stencil of each listed cell of more than SEG_SMALL blobs (sorted by
// seg_sort_listed), one CTA per cell: thread t sums the blobs t, t + RM_THREADS,
// ... of the cell (in cell order), then the CTA adds the threads' partial sums
// in a fixed tree order into part_big[16 k ..].  The cell's count is then
// replaced by -(k + 1), which is how k_rm_tile finds the table entry.
template <bool TUTTY>
__global__ void __launch_bounds__(RM_THREADS)
k_rm_stencil_big(const int32_t *__restrict__ list, const RmHead *__restrict__ hd,
                 const int32_t *__restrict__ start, int32_t *__restrict__ count,
                 const int32_t *__restrict__ perm, const double *__restrict__ x,
                 const double *__restrict__ y, const double *__restrict__ g, WParams wp,
                 double *__restrict__ part_big) {
    __shared__ double s_p[16][RM_THREADS];
    Win w;
    if (!load_win(hd, w)) return;
    const int nlist = hd->big_n;
    for (int k = blockIdx.x; k < nlist; k += gridDim.x) {
        const int64_t bc = list[k];
        const int cnt = count[bc], s0 = start[bc];
        const int64_t bx = bc / w.nby, by = bc - bx * w.nby;
        double p[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) p[q] = 0.0;
        for (int j = threadIdx.x; j < cnt; j += RM_THREADS) {
            const int32_t i = perm[s0 + j];
            const double gv = g[i];
            double wx[4], wy[4];
            blob_w8<TUTTY>(x[i], y[i], lat_x(w, bx), lat_y(w, by), wp, wx, wy);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) p[a * 4 + b] += (wx[a] * wy[b]) * gv;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) s_p[q][threadIdx.x] = p[q];
        __syncthreads();
        for (int s = RM_THREADS / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s)
#pragma unroll
                for (int q = 0; q < 16; ++q) s_p[q][threadIdx.x] += s_p[q][threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x < 16) part_big[(int64_t)k * 16 + threadIdx.x] = s_p[threadIdx.x][0];
        if (threadIdx.x == 0) count[bc] = -(k + 1);
        __syncthreads();
    }
}

struct TileOut {
    const int32_t *slot;  // output slot per output cell (EMIT)
    int64_t capacity;
    double *xo, *yo, *go;
    int64_t *ixo, *iyo;
    double *acc;    // cell values (cells mode)
    int32_t *flag;  // touched flags (cells mode)
    int64_t nrec;   // records (blobs placed): bounds-checked build
};

// The lane L of the warp whose exclusive offset off_L is the last one <= o
// (offsets non-decreasing over the lanes, off_0 = 0): the cell of blob o of
// the warp's row.  Every lane of the warp must call it.
__device__ __forceinline__ int row_owner(int off, int o) {
    int L = 0;
#pragma unroll
    for (int s = 16; s; s >>= 1) {
        const int v = __shfl_sync(0xffffffffu, off, L + s);
        if (v <= o) L += s;
    }
    return L;
}

// The 16 stencil partial sums of one base cell from its blobs in input-index
// order (the atomic ranks of k_rm_count are not reproducible, so the order is
// found here): cnt blobs, whose input index is ids(j) and whose four x
// weights times g and four y weights are wv(j, 0..7), j in [0, cnt).  Up to
// TILE_PREF indices are ordered in registers.
template <class Ids, class Wv>
__device__ __forceinline__ void cell_sums(int cnt, Ids ids_of, Wv wv, double (&p)[16]) {
    int ids[TILE_PREF];  // input indices are below 2^31
#pragma unroll
    for (int j = 0; j < TILE_PREF; ++j) ids[j] = j < cnt ? ids_of(j) : INT_MAX;
    int last = -1;
    for (int k = 0; k < cnt; ++k) {
        int best = INT_MAX;
        int bj = 0;
        if (cnt <= TILE_PREF) {
#pragma unroll
            for (int j = 0; j < TILE_PREF; ++j)
                if (ids[j] > last && ids[j] < best) {
                    best = ids[j];
                    bj = j;
                }
        } else {
            for (int j = 0; j < cnt; ++j) {
                const int v = ids_of(j);
                if (v > last && v < best) {
                    best = v;
                    bj = j;
                }
            }
        }
        last = best;
        double wxg[4], wy[4];
        wv(bj, wxg, wy);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) p[a * 4 + b] = __fma_rn(wxg[a], wy[b], p[a * 4 + b]);
    }
}

// Records of one base row (one warp) staged in shared memory with their
// weights: TW_CAP per warp; a row with more runs the per-cell walk on the
// records in HBM instead.  The row's stencil partials (16 x 32 doubles) reuse
// the first 4 KB of the same region once the row is summed.
constexpr int TW_CAP = 128;
constexpr int TW_BYTES = TW_CAP * 8 * (int)sizeof(double) + TW_CAP * (int)sizeof(int);
constexpr int TILE_SMEM = TBX * TW_BYTES;
static_assert(16 * 32 * (int)sizeof(double) <= TW_CAP * 8 * (int)sizeof(double),
              "row partials fit in the row's staging");

// One CTA per tile of TOX x TOY output cells (persistent loop over tiles).
// Warp r takes base row r of the tile, lane l its base cell l.  The row's
// blobs (contiguous runs of records, one per cell) are spread over the lanes:
// each lane forms the eight weights of one blob (all lanes busy), then each
// lane sums its own cell's blobs from shared memory in input-index order
// (16 FMA per blob).  EMIT: the new blobs are written at their slots; else the
// cell values and touched flags of every window cell go to acc / flag.
template <int WK, bool EMIT>
__global__ void __launch_bounds__(TILE_THREADS, 2)
k_rm_tile(const RmHead *hd, const int32_t *__restrict__ count,
          const int32_t *__restrict__ start, const WRec *__restrict__ recs,
          const double *__restrict__ part_big, WParams wp,
          TileOut to, double *__restrict__ mpart, RmHead *hmom) {
    extern __shared__ __align__(16) unsigned char s_tile[];
    __shared__ unsigned char s_occ[TILE_THREADS];
    __shared__ double s_mom[TILE_THREADS / 32][4];  // per warp, summed over its tiles in order
    Win w;
    if (!load_win(hd, w)) return;
    const int64_t ntx = (w.nox + TOX - 1) / TOX, nty = (w.noy + TOY - 1) / TOY;
    const int64_t ntiles = ntx * nty;
    const bool emit_ok = !EMIT || (int64_t)hd->total <= to.capacity;
    const int lbx = threadIdx.x >> 5, lby = threadIdx.x & 31;
    double *const sw = reinterpret_cast<double *>(s_tile + lbx * TW_BYTES);  // [8][TW_CAP]
    int *const sid = reinterpret_cast<int *>(sw + 8 * TW_CAP);
    if (EMIT && threadIdx.x < (TILE_THREADS / 32) * 4) s_mom[threadIdx.x >> 2][threadIdx.x & 3] = 0.0;
    // tiles are fewer than the window's cells (< 2^31): 32-bit tile indices
    const int nty32 = (int)nty;
    for (int t = blockIdx.x; t < (int)ntiles; t += gridDim.x) {
        const int tx = t / nty32, ty = t - tx * nty32;
        const int64_t ox0 = (int64_t)tx * TOX, oy0 = (int64_t)ty * TOY;
        // 1. the 16 partial sums of this thread's base cell
        {
            const int64_t bx = ox0 - 3 + lbx, by = oy0 - 3 + lby;
            double p[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) p[q] = 0.0;
            int cnt = 0;
            int64_t st = 0;
            if (bx >= 0 && bx < w.nbx && by >= 0 && by < w.nby) {
                const int64_t bc = bx * w.nby + by;
                cnt = count[bc];
                st = start[bc];
                if (cnt > 0 && !PF_IDX_OK(st + cnt - 1, to.nrec, 105)) cnt = 0;
            }
            // a tile fed by no blob touches no output cell
            if (!__syncthreads_or(cnt != 0)) {
                if (!EMIT && threadIdx.x < TOX * TOY) {
                    const int lx = threadIdx.x / TOY, ly = threadIdx.x - lx * TOY;
                    const int64_t ox = ox0 + lx, oy = oy0 + ly;
                    if (ox < w.nox && oy < w.noy) {
                        to.acc[ox * w.noy + oy] = 0.0;
                        to.flag[ox * w.noy + oy] = 0;
                    }
                }
                continue;
            }
            // the row's blobs of cells walked here (a big cell's stencil is
            // in its table): exclusive warp scan of the counts
            const int cs = cnt > 0 ? cnt : 0;
            int inc = cs;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc, o);
                if (lby >= o) inc += u;
            }
            const int off = inc - cs;
            const int total = __shfl_sync(0xffffffffu, inc, 31);
            const int64_t iy0 = cnt > 0 ? lat_y(w, by) : 0;
            // rows with at most two blobs per cell (a set near its lattice)
            // walk their cells directly: little divergence there
            const bool staged =
                total <= TW_CAP && __reduce_max_sync(0xffffffffu, (unsigned)cs) > 2u;
            if (staged) {
                const int64_t ix0 = lat_x(w, bx);
                const int st32 = (int)st;  // record positions are below 2^31
                // (a) input indices of the row's blobs (blob o of the row is
                // blob o - off[L] of the cell of lane L = row_owner(off, o))
                for (int o0 = 0; o0 < total; o0 += 32) {
                    const int o = o0 + lby;
                    const int L = row_owner(off, o);
                    const int stL = __shfl_sync(0xffffffffu, st32, L);
                    const int offL = __shfl_sync(0xffffffffu, off, L);
                    if (o < total) sid[o] = (int)recs[stL + (o - offL)].idx;
                }
                __syncwarp();
                // (b) each blob's rank in its cell by input index (indices are
                // distinct); its weights go to that position of the cell
                for (int o0 = 0; o0 < total; o0 += 32) {
                    const int o = o0 + lby;
                    const int L = row_owner(off, o);
                    const int stL = __shfl_sync(0xffffffffu, st32, L);
                    const int offL = __shfl_sync(0xffffffffu, off, L);
                    const int cntL = __shfl_sync(0xffffffffu, cs, L);
                    const int iyL = __shfl_sync(0xffffffffu, (int)iy0, L);
                    if (o < total) {
                        const int me = sid[o];
                        int r = 0;
                        for (int j = 0; j < cntL; ++j) r += sid[offL + j] < me;
                        const WRec *rc = recs + stL + (o - offL);
                        const double2 vv = *reinterpret_cast<const double2 *>(rc);
                        const double gv = rc->g;
                        double wx[4], wy[4];
                        rec_w8<WK>(vv.x, vv.y, ix0, (int64_t)iyL, wp, wx, wy);
                        const int d = offL + r;
#pragma unroll
                        for (int a = 0; a < 4; ++a) {
                            sw[a * TW_CAP + d] = wx[a] * gv;
                            sw[(4 + a) * TW_CAP + d] = wy[a];
                        }
                    }
                }
                __syncwarp();
                // (c) this lane's cell, its blobs in input-index order
                for (int k = 0; k < cnt; ++k) {
                    double wxg[4], wy[4];
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        wxg[a] = sw[a * TW_CAP + off + k];
                        wy[a] = sw[(4 + a) * TW_CAP + off + k];
                    }
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int b = 0; b < 4; ++b)
                            p[a * 4 + b] = __fma_rn(wxg[a], wy[b], p[a * 4 + b]);
                }
            } else if (cnt > 0) {  // weights per visit (sparse rows, rows above TW_CAP)
                const WRec *rc = recs + st;
                const int64_t ix0 = lat_x(w, bx);
                cell_sums(
                    cnt, [&](int j) { return (int)rc[j].idx; },
                    [&](int j, double (&wxg)[4], double (&wy)[4]) {
                        const double2 vv = *reinterpret_cast<const double2 *>(rc + j);
                        const double gv = rc[j].g;
                        double wx[4];
                        rec_w8<WK>(vv.x, vv.y, ix0, iy0, wp, wx, wy);
#pragma unroll
                        for (int a = 0; a < 4; ++a) wxg[a] = wx[a] * gv;
                    },
                    p);
            }
            if (cnt < 0) {  // a cell of more than SEG_SMALL blobs
                const double *pb = part_big + (int64_t)(-cnt - 1) * 16;
#pragma unroll
                for (int q = 0; q < 16; ++q) p[q] = pb[q];
            }
            __syncwarp();  // the row's staging is read; its partials overwrite it
            s_occ[threadIdx.x] = cnt != 0;
#pragma unroll
            for (int q = 0; q < 16; ++q) sw[q * 32 + lby] = p[q];
        }
        __syncthreads();
        // 2. each output cell: the partial sums of its 16 covering base cells,
        // in fixed (b, a) order (empty or outside cells add nothing: +0.0)
        double mom[4] = {0.0, 0.0, 0.0, 0.0};  // of the new blob this thread writes
        if (threadIdx.x < TOX * TOY) {
            const int lx = threadIdx.x / TOY, ly = threadIdx.x - lx * TOY;
            const int64_t ox = ox0 + lx, oy = oy0 + ly;
            if (ox < w.nox && oy < w.noy) {
                double sum = 0.0;
                int touched = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b)
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        const int s = (lx + 3 - a) * TBY + (ly + 3 - b);
                        if (s_occ[s]) {
                            touched = 1;
                            sum += reinterpret_cast<const double *>(
                                s_tile + (lx + 3 - a) * TW_BYTES)[(a * 4 + b) * 32 + (ly + 3 - b)];
                        }
                    }
                const int64_t cid = ox * w.noy + oy;
                if (EMIT) {
                    if (touched && emit_ok && PF_IDX_OK(to.slot[cid], to.capacity, 106)) {
                        const int64_t q = to.slot[cid];
                        const int64_t ix = lat_x(w, ox), iy = lat_y(w, oy);
                        // (ix*h + 0.5h) + xb0, each operation rounded (no FMA)
                        const double xn = __dadd_rn(__dadd_rn(__dmul_rn((double)ix, wp.h), wp.h05),
                                                    wp.xb0);
                        const double yn = __dadd_rn(__dadd_rn(__dmul_rn((double)iy, wp.h), wp.h05),
                                                    wp.yb0);
                        to.xo[q] = xn;
                        to.yo[q] = yn;
                        to.go[q] = sum;
                        add_moments(mom, xn, yn, sum);
                        if (to.ixo) to.ixo[q] = ix;
                        if (to.iyo) to.iyo[q] = iy;
                    }
                } else {
                    to.acc[cid] = sum;
                    to.flag[cid] = touched;
                }
            }
        }
        if (EMIT) {  // this tile's moments, warp by warp in a fixed order
            const int wid = threadIdx.x >> 5;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                double v = mom[q];
#pragma unroll
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if ((threadIdx.x & 31) == 0) s_mom[wid][q] += v;
            }
        }
        __syncthreads();
    }
    if (EMIT) {
        double m[4] = {0.0, 0.0, 0.0, 0.0};
        if (threadIdx.x == 0)
            for (int k = 0; k < TILE_THREADS / 32; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q) m[q] += s_mom[k][q];
        grid_moments<TILE_THREADS>(m, mpart, &hmom->ticket_out, hmom->mom + 4);
    }
}

// The tile kernels' dynamic shared memory (above the 48 KB default), set once
// per device and kernel.
template <int WK, bool EMIT>
cudaError_t tile_smem_attr() {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(k_rm_tile<WK, EMIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TILE_SMEM);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// cells mode: emit the flagged cells at their slots (cid up to the capacity;
// flags beyond the window are zero)
__global__ void __launch_bounds__(RM_THREADS)
k_rm_emit(int64_t cap_cell, const RmHead *__restrict__ hd, WParams wp,
          const int32_t *__restrict__ flag, const int32_t *__restrict__ slot,
          const double *__restrict__ acc, int64_t capacity, double *__restrict__ xo,
          double *__restrict__ yo, double *__restrict__ go, int64_t *__restrict__ ixo,
          int64_t *__restrict__ iyo) {
    Win w;
    if (!load_win(hd, w)) return;
    const int64_t cid = (int64_t)blockIdx.x * RM_THREADS + threadIdx.x;
    if (cid >= cap_cell || cid >= w.ncell) return;
    if ((int64_t)hd->total > capacity) return;  // capacity error: write nothing
    if (!flag[cid]) return;
    const int64_t ox = cid / w.noy, oy = cid - ox * w.noy;
    const int64_t ix = lat_x(w, ox), iy = lat_y(w, oy);
    const int64_t p = slot[cid];
    if (!PF_IDX_OK(p, capacity, 107)) return;
    xo[p] = __dadd_rn(__dadd_rn(__dmul_rn((double)ix, wp.h), wp.h05), wp.xb0);
    yo[p] = __dadd_rn(__dadd_rn(__dmul_rn((double)iy, wp.h), wp.h05), wp.yb0);
    go[p] = acc[cid];
    if (ixo) ixo[p] = ix;
    if (iyo) iyo[p] = iy;
}

__global__ void k_rm_finish(const RmHead *__restrict__ hd, int32_t *__restrict__ total,
                            int32_t *__restrict__ bad, int64_t *__restrict__ n_out_dev,
                            int32_t *__restrict__ status_dev, int64_t *__restrict__ window_dev,
                            double *__restrict__ moments_dev) {
    if (moments_dev)
        for (int q = 0; q < 8; ++q) moments_dev[q] = hd->mom[q];
    const int32_t t = hd->ok ? hd->total : 0;
    if (total) *total = t;
    if (bad) *bad |= hd->bad;
    if (n_out_dev) *n_out_dev = t;
    if (status_dev) *status_dev = hd->bad;
    if (window_dev) {
        int64_t ixmin = 0, iymin = 0, nbx = 0, nby = 0;
        pf::rm_head_window(*hd, ixmin, iymin, nbx, nby);
        window_dev[0] = ixmin;
        window_dev[1] = iymin;
        window_dev[2] = nbx;
        window_dev[3] = nby;
    }
}

}  // namespace

namespace pf {

// Dense-window limit: base cells <= max(2^26, 64 n).
static int64_t dense_cell_limit(int64_t n) {
    const int64_t a = (int64_t)1 << 26, b = 64 * n;
    const int64_t lim = a > b ? a : b;
    return lim < ((int64_t)1 << 30) ? lim : ((int64_t)1 << 30);
}

static int64_t big_slots(int64_t n) { return n / (SEG_SMALL + 1) + 1; }

size_t remesh_scratch_bytes(int64_t n, int64_t cap_base, int64_t cap_cell, bool cells_mode) {
    const int64_t ntA = ceil_div(cap_base, SC_TILE), ntB = ceil_div(cap_cell, SC_TILE);
    size_t b = align256(sizeof(RmHead)) + align256(4 * cap_base) + 2 * align256(4 * n) +
               align256(sizeof(WRec) * n) + align256(4 * cap_base) +
               align256(4 * cap_cell) + align256(cap_cell) +
               align256(4 * (ntA + 1)) + align256(4 * (ntB + 1)) + align256(4 * big_slots(n)) +
               align256(128 * big_slots(n)) + align256(32 * (ceil_div(n, RM_THREADS) + 1 + 2 * 1024 + 1)) +
               1024;
    if (cells_mode)
        b += align256(4 * cap_cell) + align256(8 * cap_cell) +
             align256(4 * scan_tmp_ints(cap_cell)) + popctl_scratch_bytes();
    return b;
}

pf_status remesh_core(Bump &sc, int64_t n, const double *x, const double *y, const double *g,
                      double h, double xb0, double yb0, double c, const RmWindow &win,
                      int64_t capacity, double *xo, double *yo, double *go, int64_t *ixo,
                      int64_t *iyo, int32_t *total, int32_t *bad, cudaStream_t st, int num_sms,
                      const PopCtlArgs *pc, int kernel, RmHead **head_out) {
    const bool cells = pc != nullptr;
    const int64_t cap_base = win.cap_base, cap_cell = win.cap_cell;
    if (cap_base < 1 || cap_cell < 1 || cap_cell >= ((int64_t)1 << 31)) {
        set_error("remesh: capacity %lld base / %lld output cells outside [1, 2^31)",
                  (long long)cap_base, (long long)cap_cell);
        return PF_ERR_INVALID_ARG;
    }
    // head, counts (and flags in cells mode) first: one memset zeroes them
    RmHead *hd = (RmHead *)sc.take(sizeof(RmHead));
    int32_t *count = (int32_t *)sc.take(4 * cap_base);
    int32_t *flag = cells ? (int32_t *)sc.take(4 * cap_cell) : nullptr;
    char *zero_end = cells ? (char *)(flag + cap_cell) : (char *)(count + cap_base);
    int32_t *cell = (int32_t *)sc.take(4 * n);
    int32_t *rank = (int32_t *)sc.take(4 * n);
    WRec *recs = (WRec *)sc.take(sizeof(WRec) * n);
    uint8_t *oflag = (uint8_t *)sc.take(cap_cell);
    int32_t *start = (int32_t *)sc.take(4 * cap_base);
    int32_t *slot = (int32_t *)sc.take(4 * cap_cell);
    const int64_t ntA = ceil_div(cap_base, SC_TILE), ntB = ceil_div(cap_cell, SC_TILE);
    int32_t *tsA = (int32_t *)sc.take(4 * (ntA + 1));
    int32_t *tsB = (int32_t *)sc.take(4 * (ntB + 1));
    const int64_t nbig = big_slots(n);
    int32_t *bigc = (int32_t *)sc.take(4 * nbig);
    double *part_big = (double *)sc.take(128 * nbig);
    // per-CTA moment sums of k_rm_place, then of k_rm_tile
    const int64_t gn_max = ceil_div(n, RM_THREADS) + 1, gt_max = 2 * (int64_t)num_sms + 1;
    double *mpart = (double *)sc.take(32 * (gn_max + gt_max));
    double *acc = cells ? (double *)sc.take(8 * cap_cell) : nullptr;
    int32_t *tmp = cells ? (int32_t *)sc.take(4 * scan_tmp_ints(cap_cell)) : nullptr;
    if (!mpart || (cells && !tmp)) {
        set_error("remesh: scratch too small");
        return PF_ERR_OOM;
    }
    if (head_out) *head_out = hd;
    const double h2 = 2.0 * h, h05 = 0.5 * h;
    PF_CUDA_TRY(cudaMemsetAsync(hd, 0, (size_t)(zero_end - (char *)hd), st));
    if (win.from_blobs) {
        int64_t grid = ceil_div(n, RM_THREADS);
        const int64_t cap = (int64_t)num_sms * 8;
        if (grid > cap) grid = cap;
        if (grid < 1) grid = 1;
        k_rm_extent<<<(unsigned)grid, RM_THREADS, 0, st>>>(x, y, n, xb0, yb0, h2, h05, h, hd,
                                                           cap_base, cap_cell, win.cell_limit,
                                                           cell, rank);
        PF_TRY(launch_status("k_rm_extent"));
    } else {
        if (win.nbx < 1 || win.nby < 1 || win.nbx * win.nby > cap_base ||
            (win.nbx + 3) * (win.nby + 3) > cap_cell) {
            set_error("remesh: window %lld x %lld beyond the scratch capacity", (long long)win.nbx,
                      (long long)win.nby);
            return PF_ERR_INVALID_ARG;
        }
        k_rm_set_window<<<1, 1, 0, st>>>(hd, win.ixmin, win.iymin, (int32_t)win.nbx,
                                         (int32_t)win.nby, win.rows, win.cols);
        PF_TRY(launch_status("k_rm_set_window"));
    }
    WParams wp{h, h05, xb0, yb0, xb0 / h, yb0 / h, kernel == REMESH_TUTTY ? c : c * c};
    const bool tutty = kernel == REMESH_TUTTY;
    if (n > 0) {
        const unsigned gn = (unsigned)ceil_div(n, RM_THREADS);
        k_rm_count<<<gn, RM_THREADS, 0, st>>>(x, y, n, xb0, yb0, h2, h05, h, hd, cell, rank,
                                              count, win.from_blobs);
        PF_TRY(launch_status("k_rm_count"));
        const unsigned gsc = (unsigned)(ntA + (cells ? 0 : ntB));
        k_rm_scan_up<<<gsc, SC_THREADS, 0, st>>>(hd, count, ntA, tsA, tsB, oflag);
        PF_TRY(launch_status("k_rm_scan_up"));
        k_rm_scan_down<<<gsc, SC_THREADS, 0, st>>>(hd, count, ntA, tsA, tsB, oflag, start,
                                                  slot);
        PF_TRY(launch_status("k_rm_scan_down"));
        const unsigned gp = (unsigned)std::min<int64_t>(gn, (int64_t)num_sms * 8);
        if (tutty)
            k_rm_place<true><<<gp, RM_THREADS, 0, st>>>(n, hd, cell, rank, start, x, y, g, wp,
                                                        recs, bigc, mpart);
        else
            k_rm_place<false><<<gp, RM_THREADS, 0, st>>>(n, hd, cell, rank, start, x, y, g, wp,
                                                         recs, bigc, mpart);
        PF_TRY(launch_status("k_rm_place"));
        // cells above SEG_SMALL blobs (dense clusters); the ranks are free now
        const unsigned gbig = (unsigned)std::min<int64_t>(nbig, 64);
        k_rm_big_gather<<<gbig, RM_THREADS, 0, st>>>(bigc, hd, start, count, recs, cell);
        PF_TRY(launch_status("k_rm_big_gather"));
        int32_t *perm = cell;  // the cell ids are no longer needed: sorted indices of big cells
        PF_TRY(seg_sort_listed(bigc, &hd->big_n, start, count, perm, rank, nbig, st));
        if (tutty)
            k_rm_stencil_big<true><<<gbig, RM_THREADS, 0, st>>>(bigc, hd, start, count, perm, x, y,
                                                                g, wp, part_big);
        else
            k_rm_stencil_big<false><<<gbig, RM_THREADS, 0, st>>>(bigc, hd, start, count, perm, x,
                                                                 y, g, wp, part_big);
        PF_TRY(launch_status("k_rm_stencil_big"));
    }
    {
        // persistent: two CTAs per SM, at most one per tile of the capacity
        const int64_t tiles_cap = ceil_div(cap_cell, (int64_t)TOX * TOY) + 64;
        const unsigned gt = (unsigned)std::max<int64_t>(
            1, std::min<int64_t>(std::min<int64_t>(2 * num_sms, gt_max), tiles_cap));
        TileOut to{slot, capacity, xo, yo, go, ixo, iyo, acc, flag, n};
        const int wk = tutty ? WK_TUTTY : (wp.prm == 0.0 ? WK_M4_PLAIN : WK_M4);
        double *const mp = mpart + 4 * gn_max;
#define PF_RM_TILE(K, E)                                                                  \
    do {                                                                                  \
        PF_CUDA_TRY((tile_smem_attr<K, E>()));                                            \
        k_rm_tile<K, E><<<gt, TILE_THREADS, TILE_SMEM, st>>>(hd, count, start, recs, part_big, \
                                                             wp, to, mp, hd);             \
    } while (0)
        if (cells) {
            if (wk == WK_TUTTY) PF_RM_TILE(WK_TUTTY, false);
            else if (wk == WK_M4_PLAIN) PF_RM_TILE(WK_M4_PLAIN, false);
            else PF_RM_TILE(WK_M4, false);
        } else {
            if (wk == WK_TUTTY) PF_RM_TILE(WK_TUTTY, true);
            else if (wk == WK_M4_PLAIN) PF_RM_TILE(WK_M4_PLAIN, true);
            else PF_RM_TILE(WK_M4, true);
        }
#undef PF_RM_TILE
        PF_TRY(launch_status("k_rm_tile"));
    }
    if (cells) {
        PF_TRY(popctl_decide(sc, cap_cell, acc, flag, *pc, st, &hd->ncell));
        PF_TRY(popctl_flags(cap_cell, acc, flag, pc->state, flag, st));
        PF_TRY(exclusive_scan_i32(flag, slot, cap_cell, tmp, &hd->total, st));
        k_rm_emit<<<(unsigned)ceil_div(cap_cell, RM_THREADS), RM_THREADS, 0, st>>>(
            cap_cell, hd, wp, flag, slot, acc, capacity, xo, yo, go, ixo, iyo);
        PF_TRY(launch_status("k_rm_emit"));
    }
    if (!total && !bad) return PF_OK;
    k_rm_finish<<<1, 1, 0, st>>>(hd, total, bad, nullptr, nullptr, nullptr, nullptr);
    return launch_status("k_rm_finish");
}

pf_status remesh_finish(const RmHead *hd, int64_t *n_out_dev, int32_t *status_dev,
                        int64_t *window_dev, double *moments_dev, cudaStream_t st) {
    k_rm_finish<<<1, 1, 0, st>>>(hd, nullptr, nullptr, n_out_dev, status_dev, window_dev,
                                 moments_dev);
    return launch_status("k_rm_finish");
}

}  // namespace pf

namespace {

// Common argument checks of the remesh entry points.
pf_status check_remesh_args(const char *who, int64_t n, const double *x, const double *y,
                            const double *g, double h, double xb0, double yb0, double c,
                            int64_t capacity, const double *x_out, const double *y_out,
                            const double *g_out) {
    PF_CHECK_ARG(n >= 0 && n < ((int64_t)1 << 31), "%s: n = %lld outside [0, 2^31)", who,
                 (long long)n);
    PF_CHECK_ARG(std::isfinite(h) && h > 0.0, "%s: h must be positive and finite", who);
    PF_CHECK_ARG(std::isfinite(xb0) && std::isfinite(yb0) && std::isfinite(c),
                 "%s: bounds and c must be finite", who);
    PF_CHECK_ARG(n == 0 || (x && y && g), "%s: NULL input array", who);
    PF_CHECK_ARG(capacity >= 0, "%s: negative capacity", who);
    PF_CHECK_ARG(capacity == 0 || (x_out && y_out && g_out), "%s: NULL output array", who);
    return PF_OK;
}

// Capacity in output cells for a base-cell capacity (the window's 3-cell
// border on each side; exact windows use their own (nbx + 3)(nby + 3)).
int64_t cell_cap_for(int64_t cap_base) {
    const int64_t c = cap_base + cap_base / 2 + 65536;
    return c < ((int64_t)1 << 31) - 1 ? c : ((int64_t)1 << 31) - 1;
}

// Compressed window of a sparse blob set: the sorted lattice rows holding a
// blob's base row xl or xl + 1..3, and the same for columns, built on the host
// from the blobs' left indices (read back: this path is for the rare sets
// whose dense window is too large).  The lists live in the context's own
// buffer (ctx->rm_rows), which stays valid for the call's kernels.
pf_status sparse_window(pf_ctx *ctx, int64_t n, const double *x, const double *y, double h,
                        double xb0, double yb0, int64_t limit, cudaStream_t st,
                        pf::RmWindow *win) {
    PF_TRY(pf::arena_reserve(ctx, 2 * pf::align256(4 * n)));
    int32_t *dxl = (int32_t *)pf::arena_take(ctx, 4 * n);
    int32_t *dyl = (int32_t *)pf::arena_take(ctx, 4 * n);
    k_rm_left_indices<<<(unsigned)pf::ceil_div(n, RM_THREADS), RM_THREADS, 0, st>>>(
        x, y, n, xb0, yb0, 2.0 * h, 0.5 * h, h, dxl, dyl);
    PF_TRY(pf::launch_status("k_rm_left_indices"));
    std::vector<int32_t> xl(n), yl(n);
    PF_CUDA_TRY(cudaMemcpyAsync(xl.data(), dxl, 4 * n, cudaMemcpyDeviceToHost, st));
    PF_CUDA_TRY(cudaMemcpyAsync(yl.data(), dyl, 4 * n, cudaMemcpyDeviceToHost, st));
    PF_CUDA_TRY(cudaStreamSynchronize(st));
    auto lattice = [](std::vector<int32_t> &v) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        std::vector<int32_t> r;
        r.reserve(4 * v.size());
        for (int32_t a : v)
            for (int32_t k = 0; k < 4; ++k) r.push_back(a + k);
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
        return r;
    };
    const std::vector<int32_t> rows = lattice(xl), cols = lattice(yl);
    const int64_t nbx = (int64_t)rows.size(), nby = (int64_t)cols.size();
    if (nbx * nby > limit || (nbx + 3) * (nby + 3) >= ((int64_t)1 << 31)) {
        pf::set_error("pf_remesh: the blobs touch %lld lattice rows and %lld columns; too many "
                      "for %lld blobs", (long long)nbx, (long long)nby, (long long)n);
        return PF_ERR_INVALID_ARG;
    }
    const size_t bytes = 4 * (size_t)(nbx + nby);
    if (ctx->rm_rows_cap < bytes) {
        // the previous lists may still be read by queued work of an earlier call
        PF_CUDA_TRY(cudaStreamSynchronize(st));
        if (ctx->rm_rows) PF_CUDA_TRY(cudaFree(ctx->rm_rows));
        ctx->rm_rows = nullptr;
        ctx->rm_rows_cap = 0;
        PF_CUDA_TRY(cudaMalloc(&ctx->rm_rows, bytes));
        ctx->rm_rows_cap = bytes;
    }
    int32_t *drows = static_cast<int32_t *>(ctx->rm_rows), *dcols = drows + nbx;
    PF_CUDA_TRY(cudaMemcpyAsync(drows, rows.data(), 4 * nbx, cudaMemcpyHostToDevice, st));
    PF_CUDA_TRY(cudaMemcpyAsync(dcols, cols.data(), 4 * nby, cudaMemcpyHostToDevice, st));
    PF_CUDA_TRY(cudaStreamSynchronize(st));  // the host vectors go out of scope
    *win = pf::RmWindow{false, 0, 0, nbx, nby, nbx * nby, (nbx + 3) * (nby + 3), limit};
    win->rows = drows;
    win->cols = dcols;
    return PF_OK;
}

// pf_remesh, pf_remesh_tutty and pf_remesh_population_control: window from
// the blobs on the device, remesh, optional population control of the cells
// (popctl = {gThresholdLocal, gThresholdGlobal}); one synchronisation at the
// end reads the output count.  The scratch is sized from the context's last
// window (base cells x 1.25, at least n); a window beyond it is reported by
// the device and the call runs once more on the exact window.
pf_status remesh_sync(pf_ctx *ctx, int64_t n, const double *x, const double *y, const double *g,
                      double h, double xb0, double yb0, double c, int64_t capacity,
                      double *x_out, double *y_out, double *g_out, int64_t *ix_out,
                      int64_t *iy_out, int64_t *n_out, const double *popctl, double *thr_used,
                      int kernel, void *stream) {
    PF_CHECK_ARG(ctx != nullptr, "pf_remesh: NULL context");
    PF_CHECK_ARG(n_out != nullptr, "pf_remesh: n_out is NULL");
    *n_out = 0;
    PF_TRY(check_remesh_args("pf_remesh", n, x, y, g, h, xb0, yb0, c, capacity, x_out, y_out,
                             g_out));
    if (n == 0) return PF_OK;
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t limit = pf::dense_cell_limit(n);
    pf::RmWindow win{true, 0, 0, 0, 0, 0, 0, limit};
    win.cap_base = std::min<int64_t>(std::max<int64_t>(ctx->rm_cap_base, n), limit);
    win.cap_cell = cell_cap_for(win.cap_base);
    for (int attempt = 0;; ++attempt) {
        PF_TRY(pf::arena_reserve(ctx, pf::remesh_scratch_bytes(n, win.cap_base, win.cap_cell,
                                                               popctl != nullptr) +
                                          pf::align256(sizeof(pf::PcState))));
        pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
        pf::PcState *state = (pf::PcState *)sc.take(sizeof(pf::PcState));
        pf::PopCtlArgs pc{popctl ? popctl[0] : 0.0, popctl ? popctl[1] : 0.0, state};
        pf::RmHead *hd = nullptr;
        PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, win, capacity, x_out, y_out, g_out,
                               ix_out, iy_out, nullptr, nullptr, st, ctx->num_sms,
                               popctl ? &pc : nullptr, kernel, &hd));
        PF_CUDA_TRY(cudaMemcpyAsync(ctx->host_small, hd, sizeof(pf::RmHead),
                                    cudaMemcpyDeviceToHost, st));
        if (popctl)
            PF_CUDA_TRY(cudaMemcpyAsync(ctx->host_small + 8, &state->thr, sizeof(double),
                                        cudaMemcpyDeviceToHost, st));
        PF_CUDA_TRY(cudaStreamSynchronize(st));
        pf::RmHead he;
        memcpy(&he, ctx->host_small, sizeof(he));
        if (he.bad & 1) {
            pf::set_error("pf_remesh: NaN or Inf blob coordinate");
            return PF_ERR_NAN_INPUT;
        }
        if (he.bad & 2) {
            pf::set_error("pf_remesh: blob lattice index beyond +-2^30 (coordinates far from bounds)");
            return PF_ERR_INVALID_ARG;
        }
        int64_t ixmin = 0, iymin = 0, nbx = 0, nby = 0;
        pf::rm_head_window(he, ixmin, iymin, nbx, nby);
        if (he.bad & 8) {
            if (attempt > 0) {
                pf::set_error("pf_remesh: lattice window %lld x %lld is too large for %lld blobs",
                              (long long)nbx, (long long)nby, (long long)n);
                return PF_ERR_INVALID_ARG;
            }
            if (nbx * nby > limit || (nbx + 3) * (nby + 3) >= ((int64_t)1 << 31)) {
                // a sparse set (a few blobs far from the rest): the window
                // compressed to the lattice rows and columns the blobs touch
                PF_TRY(sparse_window(ctx, n, x, y, h, xb0, yb0, limit, st, &win));
                continue;
            }
            // the exact window: no extent pass the second time
            win = pf::RmWindow{false, (int32_t)ixmin, (int32_t)iymin, nbx, nby, nbx * nby,
                               (nbx + 3) * (nby + 3), limit};
            ctx->rm_cap_base = std::min<int64_t>(nbx * nby + nbx * nby / 4, limit);
            continue;
        }
        // next calls: room for this window and 25% more (slow decay otherwise)
        ctx->rm_cap_base = std::max<int64_t>(ctx->rm_cap_base - ctx->rm_cap_base / 8,
                                             std::min<int64_t>(nbx * nby + nbx * nby / 4, limit));
        const int64_t nout = he.ok ? he.total : 0;
        *n_out = nout;
        if (popctl && thr_used) memcpy(thr_used, ctx->host_small + 8, sizeof(double));
        if (nout > capacity) {
            pf::set_error("pf_remesh: output needs %lld entries, capacity is %lld",
                          (long long)nout, (long long)capacity);
            return PF_ERR_CAPACITY;
        }
        return PF_OK;
    }
}

}  // namespace

extern "C" pf_status pf_remesh(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                               const double *g, double h, double xb0, double yb0, double c,
                               int64_t capacity, double *x_out, double *y_out, double *g_out,
                               int64_t *ix_out, int64_t *iy_out, int64_t *n_out, void *stream) {
    PF_RANGE("pf_remesh");
    pf::clear_error();
    return remesh_sync(ctx, n, x, y, g, h, xb0, yb0, c, capacity, x_out, y_out, g_out, ix_out,
                       iy_out, n_out, nullptr, nullptr, pf::REMESH_M4, stream);
}

extern "C" pf_status pf_remesh_tutty(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                     const double *g, double h, double xb0, double yb0,
                                     double hnu, int64_t capacity, double *x_out, double *y_out,
                                     double *g_out, int64_t *ix_out, int64_t *iy_out,
                                     int64_t *n_out, void *stream) {
    PF_RANGE("pf_remesh_tutty");
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
    PF_RANGE("pf_remesh_population_control");
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

extern "C" pf_status pf_remesh_async(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                     const double *g, double h, double xb0, double yb0, double c,
                                     int64_t max_base_cells, int64_t capacity, double *x_out,
                                     double *y_out, double *g_out, int64_t *ix_out,
                                     int64_t *iy_out, int64_t *n_out_dev, int32_t *status_dev,
                                     int64_t *window_dev, double *moments_dev, void *stream) {
    PF_RANGE("pf_remesh_async");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_remesh_async: NULL context");
    PF_TRY(check_remesh_args("pf_remesh_async", n, x, y, g, h, xb0, yb0, c, capacity, x_out, y_out,
                             g_out));
    PF_CHECK_ARG(max_base_cells >= 1 && max_base_cells < ((int64_t)1 << 30),
                 "pf_remesh_async: max_base_cells = %lld outside [1, 2^30)",
                 (long long)max_base_cells);
    PF_CHECK_ARG(n_out_dev != nullptr, "pf_remesh_async: n_out_dev is NULL");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t limit = std::min<int64_t>(max_base_cells, pf::dense_cell_limit(n));
    pf::RmWindow win{true, 0, 0, 0, 0, limit, cell_cap_for(limit), limit};
    PF_TRY(pf::arena_reserve(ctx, pf::remesh_scratch_bytes(n, win.cap_base, win.cap_cell, false)));
    pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
    pf::RmHead *hd = nullptr;
    PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, win, capacity, x_out, y_out, g_out,
                           ix_out, iy_out, nullptr, nullptr, st, ctx->num_sms, nullptr,
                           pf::REMESH_M4, &hd));
    return pf::remesh_finish(hd, n_out_dev, status_dev, window_dev, moments_dev, st);
}

extern "C" pf_status pf_remesh_window(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                      const double *g, double h, double xb0, double yb0, double c,
                                      int64_t ixmin, int64_t iymin, int64_t nbx, int64_t nby,
                                      int64_t capacity, double *x_out, double *y_out,
                                      double *g_out, int64_t *ix_out, int64_t *iy_out,
                                      int64_t *n_out_dev, int32_t *status_dev, void *stream) {
    PF_RANGE("pf_remesh_window");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_remesh_window: NULL context");
    PF_TRY(check_remesh_args("pf_remesh_window", n, x, y, g, h, xb0, yb0, c, capacity, x_out,
                             y_out, g_out));
    PF_CHECK_ARG(nbx > 0 && nby > 0 && nbx < ((int64_t)1 << 30) && nby < ((int64_t)1 << 30) &&
                     (nbx + 3) * (nby + 3) < ((int64_t)1 << 31),
                 "pf_remesh_window: bad window %lld x %lld", (long long)nbx, (long long)nby);
    PF_CHECK_ARG(ixmin > -((int64_t)1 << 30) && iymin > -((int64_t)1 << 30) &&
                     ixmin + nbx < ((int64_t)1 << 30) && iymin + nby < ((int64_t)1 << 30),
                 "pf_remesh_window: window outside +-2^30");
    PF_CHECK_ARG(n_out_dev != nullptr, "pf_remesh_window: n_out_dev is NULL");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const pf::RmWindow win{false, (int32_t)ixmin, (int32_t)iymin, nbx, nby, nbx * nby,
                           (nbx + 3) * (nby + 3), 0};
    PF_TRY(pf::arena_reserve(ctx, pf::remesh_scratch_bytes(n, win.cap_base, win.cap_cell, false)));
    pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
    pf::RmHead *hd = nullptr;
    PF_TRY(pf::remesh_core(sc, n, x, y, g, h, xb0, yb0, c, win, capacity, x_out, y_out, g_out,
                           ix_out, iy_out, nullptr, nullptr, st, ctx->num_sms, nullptr,
                           pf::REMESH_M4, &hd));
    return pf::remesh_finish(hd, n_out_dev, status_dev, nullptr, nullptr, st);
}
