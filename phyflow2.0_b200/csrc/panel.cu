// panel.cu -- constant-strength straight vortex panels -> velocity at points.
//
// Per pair (Katz & Plotkin 11.2.3, as _vortexPanel_Cython_cpu.pyx:374-393):
// rotate the point into the panel frame (xP, yP), panel end at (x2, 0), then
//   vxP =  g/(2pi) * theta,  theta = atan2(yP, xP-x2) - atan2(yP, xP)
//   vyP = -g/(4pi) * log((xP^2+yP^2)/((xP-x2)^2+yP^2))
// and rotate back.  Evaluated here as
//   theta = atan2(yP*x2, xP*(xP-x2) + yP^2)         (one atan2, same value in
//           (-pi, pi]: the angle between the two end-point rays)
//   log   = log1p(u), u = x2*(2xP-x2) / ((xP-x2)^2 + yP^2), while |u| < 1/2
//           (no cancellation far away), else log of the ratio itself (no
//           cancellation in 1+u next to the panel's start point)
// Geometry and accumulation in FP64, the two transcendentals in FP32.
// Panels are staged through shared memory in tiles; one target per thread.
#include "pf_common.cuh"

namespace {

constexpr int PN_THREADS = 256;
constexpr double INV_2PI = 0.15915494309189535;
constexpr double INV_4PI = 0.07957747154594767;

struct PanelSm {
    double xs, ys, c, s, x2, gam;
};

__global__ void __launch_bounds__(PN_THREADS)
k_panel_velocity(int64_t m, const double *__restrict__ gamma, const double *__restrict__ xs,
                 const double *__restrict__ ys, const double *__restrict__ xe,
                 const double *__restrict__ ye, const double *__restrict__ cosa,
                 const double *__restrict__ sina, int64_t n, const double *__restrict__ xv,
                 const double *__restrict__ yv, double *__restrict__ vx,
                 double *__restrict__ vy, int accumulate) {
    __shared__ PanelSm sp[PN_THREADS];
    const int64_t i = (int64_t)blockIdx.x * PN_THREADS + threadIdx.x;
    double px = 0.0, py = 0.0;
    if (i < n) {
        px = xv[i];
        py = yv[i];
    }
    double ax = 0.0, ay = 0.0;
    for (int64_t t0 = 0; t0 < m; t0 += PN_THREADS) {
        const int64_t j = t0 + threadIdx.x;
        __syncthreads();
        if (j < m) {
            PanelSm q;
            q.xs = xs[j];
            q.ys = ys[j];
            q.c = cosa[j];
            q.s = sina[j];
            const double lx = xe[j] - q.xs, ly = ye[j] - q.ys;
            q.x2 = q.c * lx + q.s * ly;
            q.gam = gamma[j];
            sp[threadIdx.x] = q;
        }
        __syncthreads();
        const int cnt = (int)min((int64_t)PN_THREADS, m - t0);
        for (int k = 0; k < cnt; ++k) {
            const PanelSm q = sp[k];
            const double dx = px - q.xs, dy = py - q.ys;
            const double xp = q.c * dx + q.s * dy;
            const double yp = -q.s * dx + q.c * dy;
            const double xm = xp - q.x2;
            const double a2 = xm * xm + yp * yp;
            const double num_t = yp * q.x2;
            const double den_t = xp * xm + yp * yp;
            const double num_l = q.x2 * (2.0 * xp - q.x2);
            const float theta = atan2f((float)num_t, (float)den_t);
            // log(b2/a2): log1p of u = (b2 - a2)/a2 while |u| < 1/2, else the
            // log of the FP32-rounded ratio; both ~1 ulp absolute.
            const float a2f = (float)a2;
            const float u = (float)num_l / a2f;
            const float lg = (fabsf(u) < 0.5f) ? log1pf(u) : logf((float)(xp * xp + yp * yp) / a2f);
            const double vxp = (q.gam * INV_2PI) * (double)theta;
            const double vyp = -(q.gam * INV_4PI) * (double)lg;
            ax += q.c * vxp - q.s * vyp;
            ay += q.s * vxp + q.c * vyp;
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

// Influence matrix of the panels on their collocation points
// (_vortexPanel_Cython_cpu.pyx:217-234, all in FP64 as there): A[i][j] =
// velocity induced at collocation point i by panel j at unit strength,
// projected on the tangent (cos_i, sin_i) of panel i.  One thread per (i, j),
// j fastest (coalesced rows).
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
    const double vxp = INV_2PI * (atan2(yp, xp - x2) - atan2(yp, xp));
    const double vyp = -INV_4PI * log((xp * xp + yp * yp) / ((xp - x2) * (xp - x2) + yp * yp));
    const double vx = cj * vxp - sj * vyp;
    const double vy = sj * vxp + cj * vyp;
    A[e] = vx * cosa[i] + vy * sina[i];
}

}  // namespace

extern "C" pf_status pf_panel_influence_matrix(pf_ctx *ctx, int64_t m, const double *xcp,
                                               const double *ycp, const double *xs,
                                               const double *ys, const double *xe,
                                               const double *ye, const double *cosa,
                                               const double *sina, double *A, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_panel_influence_matrix: NULL context");
    PF_CHECK_ARG(m >= 0 && m <= 32768, "pf_panel_influence_matrix: m = %lld outside [0, 32768]",
                 (long long)m);
    PF_CHECK_ARG(m == 0 || (xcp && ycp && xs && ys && xe && ye && cosa && sina && A),
                 "pf_panel_influence_matrix: NULL array");
    pf::DeviceGuard dg(ctx->device);
    if (m == 0) return PF_OK;
    k_panel_influence<<<(unsigned)pf::ceil_div(m * m, PN_THREADS), PN_THREADS, 0,
                        static_cast<cudaStream_t>(stream)>>>(m, xcp, ycp, xs, ys, xe, ye, cosa,
                                                             sina, A);
    return pf::launch_status("k_panel_influence");
}

extern "C" pf_status pf_panel_velocity(pf_ctx *ctx, int64_t m, const double *gamma,
                                       const double *xs, const double *ys, const double *xe,
                                       const double *ye, const double *cosa, const double *sina,
                                       int64_t n, const double *xv, const double *yv, double *vx,
                                       double *vy, int accumulate, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_panel_velocity: NULL context");
    PF_CHECK_ARG(m >= 0 && m <= 65536, "pf_panel_velocity: panel count %lld outside [0, 65536]",
                 (long long)m);
    PF_CHECK_ARG(n >= 0, "pf_panel_velocity: negative target count");
    PF_CHECK_ARG(m == 0 || (gamma && xs && ys && xe && ye && cosa && sina),
                 "pf_panel_velocity: NULL panel array");
    PF_CHECK_ARG(n == 0 || (xv && yv && vx && vy), "pf_panel_velocity: NULL point array");
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
    const int64_t grid = pf::ceil_div(n, PN_THREADS);
    PF_CHECK_ARG(grid <= INT32_MAX, "pf_panel_velocity: too many points");
    k_panel_velocity<<<(unsigned)grid, PN_THREADS, 0, st>>>(m, gamma, xs, ys, xe, ye, cosa, sina,
                                                           n, xv, yv, vx, vy, accumulate);
    return pf::launch_status("k_panel_velocity");
}
