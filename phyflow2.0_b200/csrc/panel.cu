// panel.cu -- constant-strength straight vortex panels -> velocity at points.
//
// Per pair (Katz & Plotkin 11.2.3, as _vortexPanel_Cython_cpu.pyx:374-393):
// rotate the point into the panel frame (xP, yP), panel end at (x2, 0), then
//   vxP =  g/(2pi) * theta,  theta = atan2(yP, xP-x2) - atan2(yP, xP)
//   vyP = -g/(4pi) * log((xP^2+yP^2)/((xP-x2)^2+yP^2))
// and rotate back.  In complex form (z = x + iy, w = vx - i vy) this is
//   w_j(z) = K_j log((z - z2_j) / (z - z1_j)),   K_j = -i g_j e^{-i alpha_j} / (2pi),
// z1 = (xs, ys), z2 = z1 + x2 e^{i alpha} (the panel end the reference's
// frame places at (x2, 0)).
//
// The panels are taken in groups of PC_G consecutive ones (a body's boundary
// is a chain, so a group is a short arc).  A group is enclosed by the circle
// |z - c| <= R around its end points' bounding-box centre, and outside it
//   sum_j w_j(z) = sum_{k>=1} A_k (R / (z - c))^k,
//   A_k = sum_j K_j (a_j^k - b_j^k) / k,  a_j = (z1_j - c)/R, b_j = (z2_j - c)/R
// (log(1 - u) = -sum u^k / k for |u| < 1; both logs have positive-real
// arguments there, so the branch is the principal one the single atan2 below
// gives).  For a point with rho = R / |z - c| <= PC_RHO the series is summed
// in FP64 to the first P terms, P the least with rho^P <= PC_EPS (1 - rho) / 2
// (remainder <= PC_EPS * rho * sum |K_j|, i.e. a relative 1e-10 of the
// group's share); nearer points take the pair formula for each panel of the
// group.  This is the reference's sum evaluated in fewer operations: every
// term it adds is kept, to 1e-10 of the group's share far away and exactly
// (up to FP32 transcendentals) near.  Nothing depends on the panel order but
// the speed: a group of scattered panels has a large R and is summed pair by
// pair for every point.
//
// The pair formula is evaluated as
//   theta = atan2(yP*x2, xP*(xP-x2) + yP^2)         (one atan2, same value in
//           (-pi, pi]: the angle between the two end-point rays)
//   log   = log1p(u), u = x2*(2xP-x2) / ((xP-x2)^2 + yP^2), while |u| < 1/2
//           (no cancellation far away), else log of the ratio itself (no
//           cancellation in 1+u next to the panel's start point)
// Geometry and accumulation in FP64, the two transcendentals in FP32.
//
// Constant-source panels (SOURCE, the reference's 'css' kernel,
// _sourcePanel_Cython_cpu.pyx:209-234 and :368-390): in the panel
// frame vxP = s/(4pi) log(r1^2/r2^2), vyP = s/(2pi) theta, i.e. the same two
// quantities with their roles exchanged; in complex form
// w = -(s/2pi) e^{-i alpha} log((z - z2)/(z - z1)), so the groups' series is
// the same with K_j = -s_j e^{-i alpha_j}/(2pi).  The source influence matrix
// projects on the normal (-sin alpha_i, cos alpha_i) instead of the tangent.
#include <algorithm>
#include <cmath>

#include "pf_common.cuh"

namespace {

constexpr int PN_THREADS = 256;
constexpr double INV_2PI = 0.15915494309189535;
constexpr double INV_4PI = 0.07957747154594767;

constexpr int PC_G = 16;           // panels per group
constexpr int PC_P = 36;           // most series terms (P at rho = PC_RHO)
constexpr double PC_RHO = 0.5;     // series used where R / |z - c| <= PC_RHO
// (measured at 2^22 points x 512 panels: rho 0.3 / 0.4 / 0.5 -> 1.82 / 1.60 /
// 1.49 ms; groups of 8 / 32 panels -> 2.26 / 2.04 ms at rho 0.4)
constexpr double PC_EPS = 1e-10;   // relative remainder of a group's share
constexpr int PC_TILE = 32;        // groups staged in shared memory at once

struct PanelSm {
    double xs, ys, c, s, x2, gam;
};

// One group: centre, radius, (R / PC_RHO)^2 and the scaled series A_1..A_P.
struct PanelGroup {
    double cx, cy, R, far_r2;
    double2 a[PC_P];
};
static_assert(sizeof(PanelGroup) % 16 == 0, "PanelGroup layout");

template <bool SOURCE>
__device__ __forceinline__ void pair_velocity(const PanelSm &q, double px, double py, double &ax,
                                              double &ay) {
    const double dx = px - q.xs, dy = py - q.ys;
    const double xp = q.c * dx + q.s * dy;
    const double yp = -q.s * dx + q.c * dy;
    const double xm = xp - q.x2;
    const double a2 = xm * xm + yp * yp;
    const double num_t = yp * q.x2;
    const double den_t = xp * xm + yp * yp;
    const double num_l = q.x2 * (2.0 * xp - q.x2);
    const float theta = atan2f((float)num_t, (float)den_t);
    // log(b2/a2): log1p of u = (b2 - a2)/a2 while |u| < 1/2, else the log of
    // the FP32-rounded ratio; both ~1 ulp absolute.
    const float a2f = (float)a2;
    const float u = (float)num_l / a2f;
    const float lg = (fabsf(u) < 0.5f) ? log1pf(u) : logf((float)(xp * xp + yp * yp) / a2f);
    const double vxp = SOURCE ? (q.gam * INV_4PI) * (double)lg : (q.gam * INV_2PI) * (double)theta;
    const double vyp = SOURCE ? (q.gam * INV_2PI) * (double)theta : -(q.gam * INV_4PI) * (double)lg;
    ax += q.c * vxp - q.s * vyp;
    ay += q.s * vxp + q.c * vyp;
}

// One warp per group: the panels' frame records, the enclosing circle and the
// series coefficients (lane k forms A_{k+1}).
template <bool SOURCE, int G = PC_G>
__global__ void __launch_bounds__(32)
k_panel_groups(int64_t m, const double *__restrict__ gamma, const double *__restrict__ xs,
               const double *__restrict__ ys, const double *__restrict__ xe,
               const double *__restrict__ ye, const double *__restrict__ cosa,
               const double *__restrict__ sina, PanelGroup *__restrict__ groups,
               PanelSm *__restrict__ pan) {
    const int64_t j0 = (int64_t)blockIdx.x * G;
    const int lane = threadIdx.x;
    const int cnt = (int)min((int64_t)G, m - j0);
    const bool has = lane < cnt;
    double x1 = 0.0, y1 = 0.0, x2e = 0.0, y2e = 0.0, kr = 0.0, ki = 0.0;
    double bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY;
    if (has) {
        const int64_t j = j0 + lane;
        PanelSm q;
        q.xs = xs[j];
        q.ys = ys[j];
        q.c = cosa[j];
        q.s = sina[j];
        const double lx = xe[j] - q.xs, ly = ye[j] - q.ys;
        q.x2 = q.c * lx + q.s * ly;
        q.gam = gamma[j];
        if (pan) pan[j] = q;
        x1 = q.xs;
        y1 = q.ys;
        x2e = q.xs + q.x2 * q.c;
        y2e = q.ys + q.x2 * q.s;
        // vortex: K = -i g e^{-i alpha}/(2 pi); source: K = -s e^{-i alpha}/(2 pi)
        kr = SOURCE ? -(q.gam * INV_2PI) * q.c : -(q.gam * INV_2PI) * q.s;
        ki = SOURCE ? (q.gam * INV_2PI) * q.s : -(q.gam * INV_2PI) * q.c;
        bx0 = fmin(x1, x2e);
        bx1 = fmax(x1, x2e);
        by0 = fmin(y1, y2e);
        by1 = fmax(y1, y2e);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bx0 = fmin(bx0, __shfl_xor_sync(0xffffffffu, bx0, o));
        bx1 = fmax(bx1, __shfl_xor_sync(0xffffffffu, bx1, o));
        by0 = fmin(by0, __shfl_xor_sync(0xffffffffu, by0, o));
        by1 = fmax(by1, __shfl_xor_sync(0xffffffffu, by1, o));
    }
    const double cx = 0.5 * (bx0 + bx1), cy = 0.5 * (by0 + by1);
    double r2 = 0.0;
    if (has) {
        const double d1 = (x1 - cx) * (x1 - cx) + (y1 - cy) * (y1 - cy);
        const double d2 = (x2e - cx) * (x2e - cx) + (y2e - cy) * (y2e - cy);
        r2 = fmax(d1, d2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
    const double R = sqrt(r2);
    const double inv = R > 0.0 ? 1.0 / R : 0.0;
    const double ar = (x1 - cx) * inv, ai = (y1 - cy) * inv;
    const double br = (x2e - cx) * inv, bi = (y2e - cy) * inv;
    // the group's scaled end points and strengths, for every lane's terms
    __shared__ double s_e[6][G];
    if (has) {
        s_e[0][lane] = ar;
        s_e[1][lane] = ai;
        s_e[2][lane] = br;
        s_e[3][lane] = bi;
        s_e[4][lane] = kr;
        s_e[5][lane] = ki;
    }
    __syncwarp();
    PanelGroup *gp = groups + blockIdx.x;
    // terms k = lane + 1 and lane + 33 (PC_P > 32 of them)
    for (int k = lane + 1; k <= PC_P; k += 32) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < cnt; ++j) {
            const double jar = s_e[0][j], jai = s_e[1][j], jbr = s_e[2][j], jbi = s_e[3][j];
            const double jkr = s_e[4][j], jki = s_e[5][j];
            double pr = 1.0, pi = 0.0, qr = 1.0, qi = 0.0;  // a^k, b^k
            for (int e = 0; e < k; ++e) {
                const double t1 = pr * jar - pi * jai;
                pi = pr * jai + pi * jar;
                pr = t1;
                const double t2 = qr * jbr - qi * jbi;
                qi = qr * jbi + qi * jbr;
                qr = t2;
            }
            const double dr = pr - qr, di = pi - qi;
            sr += jkr * dr - jki * di;
            si += jkr * di + jki * dr;
        }
        gp->a[k - 1] = make_double2(sr / k, si / k);
    }
    if (lane == 0) {
        gp->cx = cx;
        gp->cy = cy;
        gp->R = R;
        gp->far_r2 = r2 * (1.0 / (PC_RHO * PC_RHO));
    }
}

// Velocity at the points: one point per thread, the groups (series and
// panels) staged through shared memory PC_TILE at a time; a persistent grid
// keeps one staging when all groups fit one tile.
template <bool SOURCE>
__global__ void __launch_bounds__(PN_THREADS)
k_panel_velocity(int64_t ngroups, const PanelGroup *__restrict__ groups,
                 const PanelSm *__restrict__ pan, int64_t m, int64_t n,
                 const double *__restrict__ xv, const double *__restrict__ yv,
                 double *__restrict__ vx, double *__restrict__ vy, int accumulate,
                 float log2_tol) {
    __shared__ PanelGroup s_g[PC_TILE];
    __shared__ PanelSm s_p[PC_TILE * PC_G];
    const int64_t ntiles = (ngroups + PC_TILE - 1) / PC_TILE;
    bool staged = false;
    for (int64_t base = (int64_t)blockIdx.x * PN_THREADS; base < n;
         base += (int64_t)gridDim.x * PN_THREADS) {
        const int64_t i = base + threadIdx.x;
        double px = 0.0, py = 0.0;
        if (i < n) {
            px = xv[i];
            py = yv[i];
        }
        double ax = 0.0, ay = 0.0;
        for (int64_t t = 0; t < ntiles; ++t) {
            const int64_t g0 = t * PC_TILE;
            const int gc = (int)min((int64_t)PC_TILE, ngroups - g0);
            if (!staged || ntiles > 1) {
                __syncthreads();
                const double2 *srcg = reinterpret_cast<const double2 *>(groups + g0);
                double2 *dstg = reinterpret_cast<double2 *>(s_g);
                const int ng2 = gc * (int)(sizeof(PanelGroup) / 16);
                for (int e = threadIdx.x; e < ng2; e += PN_THREADS) dstg[e] = srcg[e];
                const int64_t p0 = g0 * PC_G;
                const int pc = (int)min((int64_t)PC_TILE * PC_G, m - p0);
                const double2 *srcp = reinterpret_cast<const double2 *>(pan + p0);
                double2 *dstp = reinterpret_cast<double2 *>(s_p);
                const int np2 = pc * (int)(sizeof(PanelSm) / 16);
                for (int e = threadIdx.x; e < np2; e += PN_THREADS) dstp[e] = srcp[e];
                __syncthreads();
                staged = true;
            }
            for (int c = 0; c < gc; ++c) {
                const double dx = px - s_g[c].cx, dy = py - s_g[c].cy;
                const double r2 = dx * dx + dy * dy;
                if (r2 < s_g[c].far_r2) {
                    const int j1 = (int)min((int64_t)PC_G, m - (g0 + c) * PC_G);
                    for (int j = 0; j < j1; ++j)
                        pair_velocity<SOURCE>(s_p[c * PC_G + j], px, py, ax, ay);
                } else {
                    const double R = s_g[c].R;
                    const double q = R / r2;
                    const double sr = dx * q, si = -dy * q;  // s = R / (z - c)
                    const float lr = 0.5f * __log2f((float)(R * q));
                    // at least one term (rho^2 may underflow in FP32)
                    const int P = max(1, min(PC_P, (int)ceilf(log2_tol / lr)));
                    const int Pw = __reduce_max_sync(__activemask(), P);
                    double wr = 0.0, wi = 0.0;
                    for (int k = Pw - 1; k >= 0; --k) {
                        const double2 a = s_g[c].a[k];
                        if (k < P) {
                            const double tr = fma(sr, wr, fma(-si, wi, a.x));
                            wi = fma(sr, wi, fma(si, wr, a.y));
                            wr = tr;
                        }
                    }
                    ax += sr * wr - si * wi;
                    ay -= sr * wi + si * wr;
                }
            }
        }
        if (i < n) {
            if (accumulate) {
                ax += vx[i];
                ay += vy[i];
            }
            vx[i] = ax;
            vy[i] = ay;
        }
    }
}

// ---------------------------------------------------------------------------
// Large point sets: the far groups through local expansions on a box grid.
// The points' bounding square is cut into PL_NB x PL_NB boxes.  For box b
// (centre zb, radius rb = half its diagonal) a group (c, R) is far when
// |zb - c| >= max(2R + rb, R + 2rb): then every point z of the box has
// R / |z - c| <= 1/2, inside the range where the group's series is summed to
// its stated remainder, and the series' expansion about zb converges with
// ratio |z - zb| / (|zb - c| - R) <= 1/2.  With D = zb - c and u = (z - zb)/rb,
//   sum_k A_k (R / (z - c))^k = sum_n L_n u^n,
//   L_n = (-rb / D)^n sum_{k>=1} C(n+k-1, n) A_k (R / D)^k,
// and PL_P = 40 terms leave 2^-40 of the group's share.  The box keeps the sum
// of its far groups' L_n and a bit mask of its near groups, which its points
// evaluate as before (series or the pair formula).
constexpr int PL_NB = 64;         // boxes per side of the grid
constexpr int PL_P = 40;          // local expansion terms
constexpr int64_t PL_MIN_POINTS = 32768;  // below: every group per point
constexpr int PL_MIN_GROUPS = 8;
// near groups on the box-grid path are summed by sub-groups of PL_SUB panels
// (their own series where R_sub / |z - c_sub| <= PC_RHO, else the pair formula)
constexpr int PL_SUB = 4;
static_assert(PC_G % PL_SUB == 0, "sub-groups tile a group");

struct PanelGrid {
    double x0, y0, wb;  // grid origin and box width
    unsigned long long mn[2], mx[2];  // ordered images of the points' min, max
};

__device__ __forceinline__ unsigned long long pl_ord(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double pl_unord(unsigned long long o) {
    const unsigned long long b = (o & 0x8000000000000000ull) ? (o & 0x7fffffffffffffffull) : ~o;
    return __longlong_as_double((long long)b);
}

__global__ void k_panel_grid_init(PanelGrid *gd) {
    gd->mn[0] = gd->mn[1] = ~0ull;
    gd->mx[0] = gd->mx[1] = 0ull;
}

// min / max of the point coordinates (order-preserving integer images)
__global__ void __launch_bounds__(PN_THREADS)
k_panel_bbox(int64_t n, const double *__restrict__ xv, const double *__restrict__ yv,
             PanelGrid *gd) {
    unsigned long long mnx = ~0ull, mny = ~0ull, mxx = 0ull, mxy = 0ull;
    // four points per iteration, their loads in flight together
    const int64_t stride = (int64_t)gridDim.x * PN_THREADS;
    for (int64_t i0 = (int64_t)blockIdx.x * PN_THREADS + threadIdx.x; i0 < n; i0 += 4 * stride) {
        double xs4[4], ys4[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = i0 + u * stride;
            xs4[u] = i < n ? xv[i] : xv[i0];
            ys4[u] = i < n ? yv[i] : yv[i0];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned long long ox = pl_ord(xs4[u]), oy = pl_ord(ys4[u]);
            mnx = min(mnx, ox);
            mxx = max(mxx, ox);
            mny = min(mny, oy);
            mxy = max(mxy, oy);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    // the CTA's warps, then one set of atomics per CTA
    __shared__ unsigned long long s_b[4][PN_THREADS / 32];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_b[0][wid] = mnx;
        s_b[1][wid] = mxx;
        s_b[2][wid] = mny;
        s_b[3][wid] = mxy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < PN_THREADS / 32; ++w) {
            mnx = min(mnx, s_b[0][w]);
            mxx = max(mxx, s_b[1][w]);
            mny = min(mny, s_b[2][w]);
            mxy = max(mxy, s_b[3][w]);
        }
        atomicMin(&gd->mn[0], mnx);
        atomicMax(&gd->mx[0], mxx);
        atomicMin(&gd->mn[1], mny);
        atomicMax(&gd->mx[1], mxy);
    }
}

// Boxes holding a point (the others need no local expansion); a store per
// run of equal boxes in a warp
__global__ void __launch_bounds__(PN_THREADS)
k_panel_flags(int64_t n, const double *__restrict__ xv, const double *__restrict__ yv,
              const PanelGrid *gd, int *__restrict__ flags) {
    const double x0 = gd->x0, y0 = gd->y0, wb = gd->wb;
    const int lane = threadIdx.x & 31;
    // four blocks of points per iteration, their loads in flight together
    const int64_t stride = (int64_t)gridDim.x * PN_THREADS;
    for (int64_t b0 = (int64_t)blockIdx.x * PN_THREADS; b0 < n; b0 += 4 * stride) {
        double xs4[4], ys4[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = b0 + u * stride + threadIdx.x;
            xs4[u] = i < n ? xv[i] : 0.0;
            ys4[u] = i < n ? yv[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = b0 + u * stride + threadIdx.x;
            int box = -1;
            if (i < n) {
                const int bx = min(max((int)floor((xs4[u] - x0) / wb), 0), PL_NB - 1);
                const int by = min(max((int)floor((ys4[u] - y0) / wb), 0), PL_NB - 1);
                box = bx * PL_NB + by;
            }
            const int prev = __shfl_up_sync(0xffffffffu, box, 1);
            if (box >= 0 && (lane == 0 || prev != box)) flags[box] = 1;
        }
    }
}

__global__ void k_panel_grid_set(PanelGrid *gd) {
    const double x0 = pl_unord(gd->mn[0]), x1 = pl_unord(gd->mx[0]);
    const double y0 = pl_unord(gd->mn[1]), y1 = pl_unord(gd->mx[1]);
    double e = fmax(x1 - x0, y1 - y0);
    // non-finite coordinates give no usable grid: one box holding everything
    // would be near every group, i.e. the per-point path
    if (!(e > 0.0) || !isfinite(e)) e = 1.0;
    gd->x0 = isfinite(x0) ? x0 : 0.0;
    gd->y0 = isfinite(y0) ? y0 : 0.0;
    gd->wb = e * (1.0 + 1e-9) / PL_NB;
}

// One CTA of four warps per box: the near-group mask (mwords words) and the
// local expansion of the far groups' series.  Warp v takes the far groups
// v, v + 4, ... of the box (lane n holds its partial L_n and L_{n+32}); the
// four partials are added in warp order.
__global__ void __launch_bounds__(128)
k_panel_locals(int64_t ngroups, const PanelGroup *__restrict__ groups, const PanelGrid *gd,
               const int *__restrict__ flags, int mwords, double2 *__restrict__ locals,
               unsigned *__restrict__ masks) {
    __shared__ double s_bin[PC_P][PL_P];  // [k - 1][n] = C(n + k - 1, n): lanes read rows
    __shared__ double2 s_beta[4][PC_P];   // per warp: A_k (R / D)^k
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int nn = threadIdx.x; nn < PL_P; nn += blockDim.x) {
        double c = 1.0;  // C(n, n)
        for (int k = 1; k <= PC_P; ++k) {
            s_bin[k - 1][nn] = c;
            c = c * (double)(nn + k) / (double)k;  // C(n + k, n)
        }
    }
    __shared__ double2 s_part[4][PL_P];
    const int box = blockIdx.x;
    if (!flags[box]) return;  // the whole CTA: no point there
    __syncthreads();
    const int bx = box / PL_NB, by = box - bx * PL_NB;
    const double wb = gd->wb;
    const double zbx = gd->x0 + ((double)bx + 0.5) * wb, zby = gd->y0 + ((double)by + 0.5) * wb;
    const double rb = 0.70710678118654757 * wb;
    double2 l0 = make_double2(0.0, 0.0), l1 = make_double2(0.0, 0.0);  // L_lane, L_lane+32
    for (int w = 0; w < mwords; ++w) {
        const int64_t g = (int64_t)w * 32 + lane;
        bool near = false;
        if (g < ngroups) {
            const double dx = zbx - groups[g].cx, dy = zby - groups[g].cy;
            const double R = groups[g].R;
            const double d = sqrt(dx * dx + dy * dy);
            near = !(d >= fmax(2.0 * R + rb, R + 2.0 * rb) * 1.0000001);
        }
        const unsigned nm = __ballot_sync(0xffffffffu, near);
        const unsigned valid = __ballot_sync(0xffffffffu, g < ngroups);
        if (wid == 0 && lane == 0) masks[(int64_t)box * mwords + w] = nm;
        unsigned far = valid & ~nm;
        // this warp's share: the (wid)-th, (wid + 4)-th, ... far group of the word
        for (int skip = wid; skip > 0 && far; --skip) far &= far - 1;
        while (far) {
            const int j = __ffs(far) - 1;
            far &= far - 1;
            const PanelGroup &G = groups[(int64_t)w * 32 + j];
            const double dx = zbx - G.cx, dy = zby - G.cy;
            const double inv = 1.0 / (dx * dx + dy * dy);
            const double rr = dx * inv, ri = -dy * inv;  // 1 / D
            // beta_k = A_k (R / D)^k, k = lane + 1 (and lane + 33)
            for (int k = lane + 1; k <= PC_P; k += 32) {
                double pr = 1.0, pi = 0.0, br = G.R * rr, bi = G.R * ri;
                for (int e = k; e; e >>= 1) {  // (R / D)^k by squaring
                    if (e & 1) {
                        const double t = pr * br - pi * bi;
                        pi = pr * bi + pi * br;
                        pr = t;
                    }
                    const double t = br * br - bi * bi;
                    bi = 2.0 * br * bi;
                    br = t;
                }
                const double2 a = G.a[k - 1];
                s_beta[wid][k - 1] = make_double2(a.x * pr - a.y * pi, a.x * pi + a.y * pr);
            }
            __syncwarp();
            // L_n += (-rb / D)^n sum_k C(n + k - 1, n) beta_k, for n = lane and
            // n = lane + 32 in one pass over k (even and odd k summed apart)
            const bool two = lane + 32 < PL_P;
            const int n1 = two ? lane + 32 : lane;
            double a0r = 0.0, a0i = 0.0, a1r = 0.0, a1i = 0.0;  // n = lane: even, odd k
            double c0r = 0.0, c0i = 0.0, c1r = 0.0, c1i = 0.0;  // n = lane + 32
#pragma unroll 6
            for (int k = 0; k < PC_P; k += 2) {
                const double2 b0 = s_beta[wid][k], b1 = s_beta[wid][k + 1];
                const double e0 = s_bin[k][lane], e1 = s_bin[k + 1][lane];
                a0r = fma(e0, b0.x, a0r);
                a0i = fma(e0, b0.y, a0i);
                a1r = fma(e1, b1.x, a1r);
                a1i = fma(e1, b1.y, a1i);
                const double f0 = s_bin[k][n1], f1 = s_bin[k + 1][n1];
                c0r = fma(f0, b0.x, c0r);
                c0i = fma(f0, b0.y, c0i);
                c1r = fma(f1, b1.x, c1r);
                c1i = fma(f1, b1.y, c1i);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = h ? n1 : lane;
                const double sr = h ? c0r + c1r : a0r + a1r, si = h ? c0i + c1i : a0i + a1i;
                double pr = 1.0, pi = 0.0, br = -rb * rr, bi = -rb * ri;  // (-rb / D)^n
                for (int e = n; e; e >>= 1) {
                    if (e & 1) {
                        const double t = pr * br - pi * bi;
                        pi = pr * bi + pi * br;
                        pr = t;
                    }
                    const double t = br * br - bi * bi;
                    bi = 2.0 * br * bi;
                    br = t;
                }
                const double vr = sr * pr - si * pi, vi = sr * pi + si * pr;
                if (h == 0) l0 = make_double2(l0.x + vr, l0.y + vi);
                else if (two) l1 = make_double2(l1.x + vr, l1.y + vi);
            }
            __syncwarp();  // s_beta is read before the next group refills it
            for (int skip = 3; skip > 0 && far; --skip) far &= far - 1;  // the next 3: other warps
        }
    }
    s_part[wid][lane] = l0;
    if (lane + 32 < PL_P) s_part[wid][lane + 32] = l1;
    __syncthreads();
    if (wid == 0) {
        double2 *L = locals + (int64_t)box * PL_P;
        for (int n = lane; n < PL_P; n += 32) {
            double2 v = s_part[0][n];
#pragma unroll
            for (int q = 1; q < 4; ++q) v = make_double2(v.x + s_part[q][n].x, v.y + s_part[q][n].y);
            L[n] = v;
        }
    }
}

// Velocity at the points through the box grid: the box's local expansion
// (its far groups), then its near groups one by one as k_panel_velocity does.
template <bool SOURCE>
__global__ void __launch_bounds__(PN_THREADS)
k_panel_velocity_boxed(int64_t ngroups, const PanelGroup *__restrict__ groups,
                       const PanelSm *__restrict__ pan, int64_t m, int64_t n,
                       const double *__restrict__ xv, const double *__restrict__ yv,
                       double *__restrict__ vx, double *__restrict__ vy, int accumulate,
                       float log2_tol, const PanelGrid *gd, int mwords,
                       const double2 *__restrict__ locals, const unsigned *__restrict__ masks,
                       const PanelGroup *__restrict__ subs) {
    const double x0 = gd->x0, y0 = gd->y0, wb = gd->wb;
    const double rb = 0.70710678118654757 * wb, irb = 1.0 / rb;
    for (int64_t i = (int64_t)blockIdx.x * PN_THREADS + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * PN_THREADS) {
        const double px = xv[i], py = yv[i];
        const int bx = min(max((int)floor((px - x0) / wb), 0), PL_NB - 1);
        const int by = min(max((int)floor((py - y0) / wb), 0), PL_NB - 1);
        const int box = bx * PL_NB + by;
        // the far groups: sum_n L_n u^n, u = (z - zb) / rb
        const double ur = (px - (x0 + ((double)bx + 0.5) * wb)) * irb;
        const double ui = (py - (y0 + ((double)by + 0.5) * wb)) * irb;
        const double2 *L = locals + (int64_t)box * PL_P;
        double wr = 0.0, wi = 0.0;
#pragma unroll 4
        for (int k = PL_P - 1; k >= 0; --k) {
            const double2 a = L[k];
            const double tr = fma(ur, wr, fma(-ui, wi, a.x));
            wi = fma(ur, wi, fma(ui, wr, a.y));
            wr = tr;
        }
        double ax = wr, ay = -wi;
        // the near groups
        for (int w = 0; w < mwords; ++w) {
            unsigned nm = masks[(int64_t)box * mwords + w];
            while (nm) {
                const int j = __ffs(nm) - 1;
                nm &= nm - 1;
                const int64_t g = (int64_t)w * 32 + j;
                // its sub-groups of PL_SUB panels: series or pair formulas
                const int64_t s0 = g * (PC_G / PL_SUB);
                const int64_t s1 = min(s0 + PC_G / PL_SUB, (m + PL_SUB - 1) / PL_SUB);
                for (int64_t sg = s0; sg < s1; ++sg) {
                    const PanelGroup &G = subs[sg];
                    const double dx = px - G.cx, dy = py - G.cy;
                    const double r2 = dx * dx + dy * dy;
                    if (r2 < G.far_r2) {
                        const int j1 = (int)min((int64_t)PL_SUB, m - sg * PL_SUB);
                        for (int q = 0; q < j1; ++q)
                            pair_velocity<SOURCE>(pan[sg * PL_SUB + q], px, py, ax, ay);
                    } else {
                        const double R = G.R;
                        const double q = R / r2;
                        const double sr = dx * q, si = -dy * q;  // s = R / (z - c)
                        const float lr = 0.5f * __log2f((float)(R * q));
                        const int P = max(1, min(PC_P, (int)ceilf(log2_tol / lr)));
                        double tr0 = 0.0, ti0 = 0.0;
                        for (int k = P - 1; k >= 0; --k) {
                            const double2 a = G.a[k];
                            const double t = fma(sr, tr0, fma(-si, ti0, a.x));
                            ti0 = fma(sr, ti0, fma(si, tr0, a.y));
                            tr0 = t;
                        }
                        ax += sr * tr0 - si * ti0;
                        ay -= sr * ti0 + si * tr0;
                    }
                }
            }
        }
        if (accumulate) {
            ax += vx[i];
            ay += vy[i];
        }
        vx[i] = ax;
        vy[i] = ay;
    }
}

// Influence matrix of the panels on their collocation points
// (_vortexPanel_Cython_cpu.pyx:217-234, all in FP64 as there): A[i][j] =
// velocity induced at collocation point i by panel j at unit strength,
// projected on the tangent (cos_i, sin_i) of panel i.  One thread per (i, j),
// j fastest (coalesced rows).  SOURCE: source panels
// (_sourcePanel_Cython_cpu.pyx:209-234), projected on the normal
// (-sin_i, cos_i).
template <bool SOURCE>
__global__ void __launch_bounds__(PN_THREADS)
k_panel_influence(int64_t m, const double *__restrict__ xcp, const double *__restrict__ ycp,
                  const double *__restrict__ xs, const double *__restrict__ ys,
                  const double *__restrict__ xe, const double *__restrict__ ye,
                  const double *__restrict__ cosa, const double *__restrict__ sina,
                  double *__restrict__ A) {
    const int64_t e = (int64_t)blockIdx.x * PN_THREADS + threadIdx.x;
    if (e >= m * m) return;
    const int64_t i = e / m, j = e - i * m;
    const double cj = cosa[j], sj = sina[j];
    const double lx = xe[j] - xs[j], ly = ye[j] - ys[j];
    const double x2 = cj * lx + sj * ly;
    const double dx = xcp[i] - xs[j], dy = ycp[i] - ys[j];
    const double xp = cj * dx + sj * dy;
    const double yp = -sj * dx + cj * dy;
    const double th = atan2(yp, xp - x2) - atan2(yp, xp);
    const double lg = log((xp * xp + yp * yp) / ((xp - x2) * (xp - x2) + yp * yp));
    const double vxp = SOURCE ? INV_4PI * lg : INV_2PI * th;
    const double vyp = SOURCE ? INV_2PI * th : -INV_4PI * lg;
    const double vx = cj * vxp - sj * vyp;
    const double vy = sj * vxp + cj * vyp;
    A[e] = SOURCE ? vx * -sina[i] + vy * cosa[i] : vx * cosa[i] + vy * sina[i];
}

}  // namespace

static pf_status influence_matrix(pf_ctx *ctx, const char *name, int64_t m, const double *xcp,
                                  const double *ycp, const double *xs, const double *ys,
                                  const double *xe, const double *ye, const double *cosa,
                                  const double *sina, double *A, void *stream, bool source) {
    PF_CHECK_ARG(ctx != nullptr, "%s: NULL context", name);
    PF_CHECK_ARG(m >= 0 && m <= 32768, "%s: m = %lld outside [0, 32768]", name, (long long)m);
    PF_CHECK_ARG(m == 0 || (xcp && ycp && xs && ys && xe && ye && cosa && sina && A),
                 "%s: NULL array", name);
    pf::DeviceGuard dg(ctx->device);
    if (m == 0) return PF_OK;
    const unsigned grid = (unsigned)pf::ceil_div(m * m, PN_THREADS);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (source)
        k_panel_influence<true><<<grid, PN_THREADS, 0, st>>>(m, xcp, ycp, xs, ys, xe, ye, cosa,
                                                             sina, A);
    else
        k_panel_influence<false><<<grid, PN_THREADS, 0, st>>>(m, xcp, ycp, xs, ys, xe, ye, cosa,
                                                              sina, A);
    return pf::launch_status("k_panel_influence");
}

static pf_status panel_velocity(pf_ctx *ctx, const char *name, int64_t m, const double *gamma,
                                const double *xs, const double *ys, const double *xe,
                                const double *ye, const double *cosa, const double *sina,
                                int64_t n, const double *xv, const double *yv, double *vx,
                                double *vy, int accumulate, void *stream, bool source) {
    PF_CHECK_ARG(ctx != nullptr, "%s: NULL context", name);
    PF_CHECK_ARG(m >= 0 && m <= 65536, "%s: panel count %lld outside [0, 65536]", name,
                 (long long)m);
    PF_CHECK_ARG(n >= 0, "%s: negative target count", name);
    PF_CHECK_ARG(m == 0 || (gamma && xs && ys && xe && ye && cosa && sina),
                 "%s: NULL panel array", name);
    PF_CHECK_ARG(n == 0 || (xv && yv && vx && vy), "%s: NULL point array", name);
    pf::DeviceGuard dg(ctx->device);
    if (n == 0) return PF_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (m == 0) {
        if (!accumulate) {
            PF_CUDA_TRY(cudaMemsetAsync(vx, 0, sizeof(double) * n, st));
            PF_CUDA_TRY(cudaMemsetAsync(vy, 0, sizeof(double) * n, st));
        }
        return PF_OK;
    }
    const int64_t ngroups = pf::ceil_div(m, PC_G);
    const size_t gbytes = sizeof(PanelGroup) * (size_t)ngroups;
    const size_t pbytes = sizeof(PanelSm) * (size_t)m;
    // large point sets take the far groups through the box grid's local
    // expansions
    const bool boxed = n >= PL_MIN_POINTS && ngroups >= PL_MIN_GROUPS;
    const int mwords = (int)pf::ceil_div(ngroups, (int64_t)32);
    const size_t lbytes = boxed ? sizeof(double2) * PL_P * PL_NB * PL_NB : 0;
    const size_t mbytes = boxed ? sizeof(unsigned) * (size_t)mwords * PL_NB * PL_NB : 0;
    const size_t fbytes = boxed ? sizeof(int) * PL_NB * PL_NB : 0;
    const int64_t nsubs = pf::ceil_div(m, (int64_t)PL_SUB);
    const size_t sbytes = boxed ? sizeof(PanelGroup) * (size_t)nsubs : 0;
    PF_TRY(pf::arena_reserve(ctx, pf::align256(gbytes) + pf::align256(pbytes) +
                                      (boxed ? pf::align256(sizeof(PanelGrid)) +
                                                   pf::align256(lbytes) + pf::align256(mbytes) +
                                                   pf::align256(fbytes) + pf::align256(sbytes)
                                             : 0)));
    auto *groups = static_cast<PanelGroup *>(pf::arena_take(ctx, gbytes));
    auto *pan = static_cast<PanelSm *>(pf::arena_take(ctx, pbytes));
    PanelGrid *gd = nullptr;
    double2 *locals = nullptr;
    unsigned *masks = nullptr;
    int *flags = nullptr;
    PanelGroup *subs = nullptr;
    if (boxed) {
        gd = static_cast<PanelGrid *>(pf::arena_take(ctx, sizeof(PanelGrid)));
        locals = static_cast<double2 *>(pf::arena_take(ctx, lbytes));
        masks = static_cast<unsigned *>(pf::arena_take(ctx, mbytes));
        flags = static_cast<int *>(pf::arena_take(ctx, fbytes));
        subs = static_cast<PanelGroup *>(pf::arena_take(ctx, sbytes));
    }
    if (!groups || !pan || (boxed && (!gd || !locals || !masks || !flags || !subs))) {
        pf::set_error("%s: scratch too small", name);
        return PF_ERR_OOM;
    }
    if (source)
        k_panel_groups<true><<<(unsigned)ngroups, 32, 0, st>>>(m, gamma, xs, ys, xe, ye, cosa,
                                                               sina, groups, pan);
    else
        k_panel_groups<false><<<(unsigned)ngroups, 32, 0, st>>>(m, gamma, xs, ys, xe, ye, cosa,
                                                                sina, groups, pan);
    PF_TRY(pf::launch_status("k_panel_groups"));
    // persistent grid: a few CTAs per SM, each over many blocks of points
    const int64_t grid = std::min<int64_t>(pf::ceil_div(n, PN_THREADS), (int64_t)ctx->num_sms * 4);
    // P = ceil(log2(PC_EPS (1 - PC_RHO) / 2) / log2(rho)) terms for rho <= PC_RHO
    const float log2_tol = (float)std::log2(PC_EPS * (1.0 - PC_RHO) / 2.0);
    if (boxed) {
        if (source)
            k_panel_groups<true, PL_SUB><<<(unsigned)nsubs, 32, 0, st>>>(
                m, gamma, xs, ys, xe, ye, cosa, sina, subs, nullptr);
        else
            k_panel_groups<false, PL_SUB><<<(unsigned)nsubs, 32, 0, st>>>(
                m, gamma, xs, ys, xe, ye, cosa, sina, subs, nullptr);
        PF_TRY(pf::launch_status("k_panel_groups"));
        k_panel_grid_init<<<1, 1, 0, st>>>(gd);
        PF_TRY(pf::launch_status("k_panel_grid_init"));
        k_panel_bbox<<<(unsigned)grid, PN_THREADS, 0, st>>>(n, xv, yv, gd);
        PF_TRY(pf::launch_status("k_panel_bbox"));
        k_panel_grid_set<<<1, 1, 0, st>>>(gd);
        PF_TRY(pf::launch_status("k_panel_grid_set"));
        PF_CUDA_TRY(cudaMemsetAsync(flags, 0, fbytes, st));
        k_panel_flags<<<(unsigned)grid, PN_THREADS, 0, st>>>(n, xv, yv, gd, flags);
        PF_TRY(pf::launch_status("k_panel_flags"));
        k_panel_locals<<<PL_NB * PL_NB, 128, 0, st>>>(ngroups, groups, gd, flags, mwords, locals,
                                                      masks);
        PF_TRY(pf::launch_status("k_panel_locals"));
        if (source)
            k_panel_velocity_boxed<true><<<(unsigned)grid, PN_THREADS, 0, st>>>(
                ngroups, groups, pan, m, n, xv, yv, vx, vy, accumulate, log2_tol, gd, mwords,
                locals, masks, subs);
        else
            k_panel_velocity_boxed<false><<<(unsigned)grid, PN_THREADS, 0, st>>>(
                ngroups, groups, pan, m, n, xv, yv, vx, vy, accumulate, log2_tol, gd, mwords,
                locals, masks, subs);
        return pf::launch_status("k_panel_velocity_boxed");
    }
    if (source)
        k_panel_velocity<true><<<(unsigned)grid, PN_THREADS, 0, st>>>(
            ngroups, groups, pan, m, n, xv, yv, vx, vy, accumulate, log2_tol);
    else
        k_panel_velocity<false><<<(unsigned)grid, PN_THREADS, 0, st>>>(
            ngroups, groups, pan, m, n, xv, yv, vx, vy, accumulate, log2_tol);
    return pf::launch_status("k_panel_velocity");
}

extern "C" pf_status pf_panel_influence_matrix(pf_ctx *ctx, int64_t m, const double *xcp,
                                               const double *ycp, const double *xs,
                                               const double *ys, const double *xe,
                                               const double *ye, const double *cosa,
                                               const double *sina, double *A, void *stream) {
    PF_RANGE("pf_panel_influence_matrix");
    pf::clear_error();
    return influence_matrix(ctx, "pf_panel_influence_matrix", m, xcp, ycp, xs, ys, xe, ye, cosa,
                            sina, A, stream, false);
}

extern "C" pf_status pf_source_panel_influence_matrix(pf_ctx *ctx, int64_t m, const double *xcp,
                                                      const double *ycp, const double *xs,
                                                      const double *ys, const double *xe,
                                                      const double *ye, const double *cosa,
                                                      const double *sina, double *A,
                                                      void *stream) {
    PF_RANGE("pf_source_panel_influence_matrix");
    pf::clear_error();
    return influence_matrix(ctx, "pf_source_panel_influence_matrix", m, xcp, ycp, xs, ys, xe, ye,
                            cosa, sina, A, stream, true);
}

extern "C" pf_status pf_panel_velocity(pf_ctx *ctx, int64_t m, const double *gamma,
                                       const double *xs, const double *ys, const double *xe,
                                       const double *ye, const double *cosa, const double *sina,
                                       int64_t n, const double *xv, const double *yv, double *vx,
                                       double *vy, int accumulate, void *stream) {
    PF_RANGE("pf_panel_velocity");
    pf::clear_error();
    return panel_velocity(ctx, "pf_panel_velocity", m, gamma, xs, ys, xe, ye, cosa, sina, n, xv,
                          yv, vx, vy, accumulate, stream, false);
}

extern "C" pf_status pf_source_panel_velocity(pf_ctx *ctx, int64_t m, const double *sigma,
                                              const double *xs, const double *ys,
                                              const double *xe, const double *ye,
                                              const double *cosa, const double *sina, int64_t n,
                                              const double *xv, const double *yv, double *vx,
                                              double *vy, int accumulate, void *stream) {
    PF_RANGE("pf_source_panel_velocity");
    pf::clear_error();
    return panel_velocity(ctx, "pf_source_panel_velocity", m, sigma, xs, ys, xe, ye, cosa, sina,
                          n, xv, yv, vx, vy, accumulate, stream, true);
}
