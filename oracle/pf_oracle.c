/*
 * pf_oracle.c -- CPU restatement of the pHyFlow vortex-blob hot path, FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it to produce the
 * FP64 answer that the CUDA path is compared against.  The product library
 * never links, loads or calls it, and there is no CPU fallback built on it.
 *
 * Every function restates the reference algorithm in our own code and cites
 * the reference file:line it follows (paths are relative to the pHyFlow
 * source tree).  Compile with -ffp-contract=off so that the operation order
 * written here is the one executed (the reference is built without FMA).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.141592653589793

/* Gaussian-blob Biot-Savart velocity by direct summation.
 * Follows src/cpp/blobs/c/vv2parGauss_C/vv2parGauss_C_cpu.c:100-153 and the
 * identical Cython kernel src/cpp/blobs/cython/vv2parGauss_Cython/
 * vv2parGauss_Cython_cpu.pyx:82-102:
 *   r2 = dx*dx + dy*dy + 1e-12
 *   s  = (g/r2) * (1 - exp(-r2/ksigmasqr))
 *   vx -= dy*s ; vy += dx*s ; both scaled by 1/(2 pi) at the end.
 * OpenMP over targets, as the reference. */
void or_velocity_direct_gauss(int64_t ns, const double *xs, const double *ys,
                              const double *gs, int64_t nt, const double *xt,
                              const double *yt, double ksigmasqr, double *vx,
                              double *vy, int nthreads)
{
    const double EPS = 1e-12;
    const double inv_2pi = 0.5 / OR_PI;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t k = 0; k < nt; ++k) {
        const double xk = xt[k], yk = yt[k];
        double ax = 0.0, ay = 0.0;
        for (int64_t m = 0; m < ns; ++m) {
            const double dx = xk - xs[m];
            const double dy = yk - ys[m];
            const double r2 = dx * dx + dy * dy + EPS;
            const double s = (gs[m] / r2) * (1.0 - exp(-r2 / ksigmasqr));
            ax -= dy * s;
            ay += dx * s;
        }
        vx[k] = inv_2pi * ax;
        vy[k] = inv_2pi * ay;
    }
}

/* Induced vorticity of Gaussian blobs: restates ww2parGauss_C_cpu
 * (src/cpp/blobs/c/ww2parGauss_C/ww2parGauss_C_cpu.c:131-145):
 *   w_k = (1/pi) sum_m g_m exp(-(dx^2 + dy^2 + 1e-12)/ksigmasqr) / ksigmasqr */
void or_vorticity_direct_gauss(int64_t ns, const double *xs, const double *ys,
                               const double *gs, int64_t nt, const double *xt,
                               const double *yt, double ksigmasqr, double *w, int nthreads)
{
    const double EPS = 1e-12;
    const double inv_pi = 1.0 / OR_PI;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t k = 0; k < nt; ++k) {
        double wk = 0.0;
        for (int64_t m = 0; m < ns; ++m) {
            const double dx = xt[k] - xs[m];
            const double dy = yt[k] - ys[m];
            const double r2 = dx * dx + dy * dy + EPS;
            wk += gs[m] * exp(-r2 / ksigmasqr);
        }
        w[k] = inv_pi * wk / ksigmasqr;
    }
}

/* Cutoff-kernel velocity by direct summation: restates vv2par_C_cpu
 * (src/cpp/blobs/c/vv2par_C/vv2par_C_cpu.c:135-151) and the Cython twin
 * (src/cpp/blobs/cython/vv2par_Cython/vv2par_Cython_cpu.pyx):
 *   r2 = dx*dx + dy*dy + sigmasqr ;  s = g/r2 ;  vx -= dy*s ; vy += dx*s
 * then both scaled by 1/(2 pi). */
void or_velocity_direct_cutoff(int64_t ns, const double *xs, const double *ys,
                               const double *gs, int64_t nt, const double *xt,
                               const double *yt, double sigmasqr, double *vx,
                               double *vy, int nthreads)
{
    const double inv_2pi = 0.5 / OR_PI;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t k = 0; k < nt; ++k) {
        double ax = 0.0, ay = 0.0;
        for (int64_t m = 0; m < ns; ++m) {
            const double dx = xt[k] - xs[m];
            const double dy = yt[k] - ys[m];
            const double r2 = dx * dx + dy * dy + sigmasqr;
            const double s = gs[m] / r2;
            ax -= dy * s;
            ay += dx * s;
        }
        vx[k] = inv_2pi * ax;
        vy[k] = inv_2pi * ay;
    }
}

/* Cutoff-kernel induced vorticity as the reference computes it: restates
 * ww2par_C_cpu (src/cpp/blobs/c/ww2par_C/ww2par_C_cpu.c:132-145):
 *   w_k = (1/(2 pi)) sum_m g_m / sqrt(dx^2 + dy^2 + sigmasqr) */
void or_vorticity_direct_cutoff(int64_t ns, const double *xs, const double *ys,
                                const double *gs, int64_t nt, const double *xt,
                                const double *yt, double sigmasqr, double *w, int nthreads)
{
    const double inv_2pi = 0.5 / OR_PI;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t k = 0; k < nt; ++k) {
        double wk = 0.0;
        for (int64_t m = 0; m < ns; ++m) {
            const double dx = xt[k] - xs[m];
            const double dy = yt[k] - ys[m];
            wk += gs[m] / sqrt(dx * dx + dy * dy + sigmasqr);
        }
        w[k] = inv_2pi * wk;
    }
}

/* Constant-strength straight vortex panels, induced velocity at points.
 * Follows src/cpp/panels/cython/vortexPanel_Cython/_vortexPanel_Cython_cpu.pyx
 * :352-393 (Katz & Plotkin 11.2.3): rotate the point into the panel frame,
 *   vxP =  g/(2pi) (atan2(yP, xP-x2) - atan2(yP, xP))
 *   vyP = -g/(4pi) log((xP^2+yP^2)/((xP-x2)^2+yP^2))
 * and rotate back. */
void or_panel_velocity(int64_t m, const double *gamma, const double *xs,
                       const double *ys, const double *xe, const double *ye,
                       const double *cosa, const double *sina, int64_t n,
                       const double *xv, const double *yv, double *vx,
                       double *vy, int nthreads)
{
    const double inv_2pi = 1.0 / (2.0 * OR_PI);
    const double inv_4pi = inv_2pi / 2.0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < n; ++i) {
        double ax = 0.0, ay = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            const double Lx = xe[j] - xs[j];
            const double Ly = ye[j] - ys[j];
            const double x2 = cosa[j] * Lx + sina[j] * Ly;
            const double xP = cosa[j] * (xv[i] - xs[j]) + sina[j] * (yv[i] - ys[j]);
            const double yP = -sina[j] * (xv[i] - xs[j]) + cosa[j] * (yv[i] - ys[j]);
            const double vxP = (gamma[j] * inv_2pi) * (atan2(yP, (xP - x2)) - atan2(yP, xP));
            const double vyP = -(gamma[j] * inv_4pi) *
                               log((xP * xP + yP * yP) / ((xP - x2) * (xP - x2) + yP * yP));
            ax += cosa[j] * vxP - sina[j] * vyP;
            ay += sina[j] * vxP + cosa[j] * vyP;
        }
        vx[i] = ax;
        vy[i] = ay;
    }
}

/* Constant-strength source panels, induced velocity at points.  Follows
 * src/cpp/panels/cython/sourcePanel_Cython/_sourcePanel_Cython_cpu.pyx
 * :368-390: in the panel frame
 *   vxP = s/(4pi) log((xP^2+yP^2)/((xP-x2)^2+yP^2))
 *   vyP = s/(2pi) (atan2(yP, xP-x2) - atan2(yP, xP))
 * and rotate back. */
void or_source_panel_velocity(int64_t m, const double *sigma, const double *xs,
                              const double *ys, const double *xe, const double *ye,
                              const double *cosa, const double *sina, int64_t n,
                              const double *xv, const double *yv, double *vx,
                              double *vy, int nthreads)
{
    const double inv_2pi = 1.0 / (2.0 * OR_PI);
    const double inv_4pi = inv_2pi / 2.0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < n; ++i) {
        double ax = 0.0, ay = 0.0;
        for (int64_t j = 0; j < m; ++j) {
            const double Lx = xe[j] - xs[j];
            const double Ly = ye[j] - ys[j];
            const double x2 = cosa[j] * Lx + sina[j] * Ly;
            const double xP = cosa[j] * (xv[i] - xs[j]) + sina[j] * (yv[i] - ys[j]);
            const double yP = -sina[j] * (xv[i] - xs[j]) + cosa[j] * (yv[i] - ys[j]);
            const double vxP = (sigma[j] * inv_4pi) *
                               log((xP * xP + yP * yP) / ((xP - x2) * (xP - x2) + yP * yP));
            const double vyP = (sigma[j] * inv_2pi) * (atan2(yP, (xP - x2)) - atan2(yP, xP));
            ax += cosa[j] * vxP - sina[j] * vyP;
            ay += sina[j] * vxP + cosa[j] * vyP;
        }
        vx[i] = ax;
        vy[i] = ay;
    }
}

/* One-dimensional M4' interpolation weights with the Wee diffusion term c^2.
 * Follows src/cpp/blobs/c++/interpolation_kernels_1d/
 * _interpolation_kernels_1d.cpp:75-89, including its branch structure: the
 * outer interval is open on both ends and |x| == 1 falls through to 0. */
void or_m4prime(int64_t n, const double *x, double c, double *w)
{
    for (int64_t k = 0; k < n; ++k) {
        const double a = fabs(x[k]);
        if (a > 1.0 && a < 2.0) {
            w[k] = 0.5 * pow(2.0 - a, 2.0) * (1.0 - a) -
                   pow(c, 2.0) * pow(2.0 - a, 2.0) * (1.0 - 2.0 * a);
        } else if (a >= 0.0 && a < 1.0) {
            w[k] = 1.0 - 2.5 * pow(x[k], 2.0) + 1.5 * pow(a, 3.0) -
                   pow(c, 2.0) * (2.0 - 9.0 * pow(x[k], 2) + 6.0 * pow(a, 3.0));
        } else {
            w[k] = 0.0;
        }
    }
}

/* Left/bottom index of the 4x4 remesh window of each blob.
 * Follows src/python/blobs/base/regrid/_regridding.py:157-158:
 *   xL = int64(ceil((x - xB0 - 2.0*h + 0.5*h)/h)) - 1
 * evaluated left to right as numpy does. */
void or_remesh_left_index(int64_t n, const double *x, double b0, double h,
                          int64_t *il)
{
    const double h2 = 2.0 * h, h05 = 0.5 * h;
    for (int64_t k = 0; k < n; ++k) {
        const double t = ((x[k] - b0) - h2) + h05;
        il[k] = (int64_t)ceil(t / h) - 1;
    }
}

/* Sum of g, g*x and g*y in FP64 (circulation and linear impulse), and sum
 * of |g|, used by the conservation checks. Plain sequential order. */
void or_moments(int64_t n, const double *x, const double *y, const double *g,
                double *out4)
{
    double s0 = 0.0, sx = 0.0, sy = 0.0, sa = 0.0;
    for (int64_t k = 0; k < n; ++k) {
        s0 += g[k];
        sx += g[k] * x[k];
        sy += g[k] * y[k];
        sa += fabs(g[k]);
    }
    out4[0] = s0;
    out4[1] = sx;
    out4[2] = sy;
    out4[3] = sa;
}
