// gauss_pair.cuh -- the Gaussian-blob pair interaction in FP32, shared by the
// direct sum and the FMM near field.
//
// Kernel (src/cpp/blobs/c/vv2parGauss_C/vv2parGauss_C_cpu.c:146-150):
//   r2 = dx^2 + dy^2 + 1e-12;  s = g/r2 * (1 - exp(-r2/ksigmasqr))
//   vx -= dy*s;  vy += dx*s
//
// FP32 evaluation:
// * dx, dy come from hi/lo float pairs: (t_hi - s_hi) + (t_lo - s_lo); the hi
//   difference is exact for nearby pairs (Sterbenz), so positions keep ~48 bits.
// * exp via ex2.approx (MUFU), 1/r2 via rcp.approx (MUFU).
// * 1 - exp(-x) cancels for small x = r2/ksigmasqr; below X_SERIES it is
//   replaced by its Taylor series x(1 - x/2 + x^2/6 - ...) to x^6, whose
//   truncation error at x = X_SERIES is below 5e-8 relative.
// * Where r2 * log2(e)/ksigmasqr >= Y_FAR = 26, ex2 returns below 2^-25 and
//   1 - ex2(...) rounds to 1.0f exactly, so s = g * rcp(r2) bitwise: callers
//   that know every pair of a tile lies that far (pair2_far) skip the ex2.
#pragma once
#include "pf_common.cuh"

namespace pfd {

constexpr float X_SERIES = 0.25f;
constexpr double Y_FAR = 26.0;
constexpr float LOG2E_F = 1.4426950408889634f;

struct GaussParams {
    float c_t;       // -log2(e)/ksigmasqr  (argument of ex2)
    float c_x;       // 1/ksigmasqr
    float r2_series; // X_SERIES * ksigmasqr
    float r2_far;    // Y_FAR * ksigmasqr / log2(e): beyond it 1 - exp(-x) is 1.0f
};

__host__ __device__ inline GaussParams make_gauss_params(double ksigmasqr) {
    GaussParams p;
    p.c_t = (float)(-1.4426950408889634 / ksigmasqr);
    p.c_x = (float)(1.0 / ksigmasqr);
    p.r2_series = (float)(0.25 * ksigmasqr);
    p.r2_far = (float)(Y_FAR / 1.4426950408889634 * ksigmasqr);
    return p;
}

// (1 - exp(-x)) / r2 * g given r2, with the series branch for small x
// (SERIES = false: caller guarantees r2 >= r2_series).
template <bool SERIES = true>
__device__ __forceinline__ float gauss_s(float r2, float g, const GaussParams &p) {
    float e = ex2_approx(r2 * p.c_t);
    float om = 1.0f - e;
    if (SERIES && r2 < p.r2_series) {
        float x = r2 * p.c_x;
        float q = fmaf(x, -1.0f / 720.0f, 1.0f / 120.0f);
        q = fmaf(x, q, -1.0f / 24.0f);
        q = fmaf(x, q, 1.0f / 6.0f);
        q = fmaf(x, q, -0.5f);
        q = fmaf(x, q, 1.0f);
        om = x * q;
    }
    return g * om * rcp_approx(r2);
}


// ---------------------------------------------------------------------------
// Two targets against one source with Blackwell's packed f32x2 arithmetic.
// A 64-bit register holds (target a, target b); every packed operation is the
// element-wise IEEE round-to-nearest operation, in the same order as the
// scalar code above, so each lane's two results are bitwise those of two
// scalar evaluations.  Only ex2 and rcp (MUFU) stay scalar.
//
// Source layout in shared memory (broadcast form, so loads land directly in
// packed registers):  hi = {x_hi, x_hi, y_hi, y_hi}, lo = {x_lo, x_lo, y_lo,
// y_lo} (two ulonglong2), g2 = {g, g}.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pack2(float a, float b) {
    f32x2 d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ void unpack2(f32x2 v, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

struct GaussParams2 {
    f32x2 c_t, c_x, eps, one;
    float r2_series, c_x1;
};

__device__ __forceinline__ GaussParams2 make_params2(const GaussParams &p) {
    GaussParams2 q;
    q.c_t = pack2(p.c_t, p.c_t);
    q.c_x = pack2(p.c_x, p.c_x);
    q.eps = pack2(1e-12f, 1e-12f);
    q.one = pack2(1.0f, 1.0f);
    q.r2_series = p.r2_series;
    q.c_x1 = p.c_x;
    return q;
}

__device__ __forceinline__ float series_om(float r2, float c_x) {
    const float x = r2 * c_x;
    float q = fmaf(x, -1.0f / 720.0f, 1.0f / 120.0f);
    q = fmaf(x, q, -1.0f / 24.0f);
    q = fmaf(x, q, 1.0f / 6.0f);
    q = fmaf(x, q, -0.5f);
    q = fmaf(x, q, 1.0f);
    return x * q;
}

// Accumulates, for targets (a, b): nx += dy*s, ny += dx*s  (note the sign:
// the x velocity is -nx; negation is exact, so -nx equals the scalar sum).
// SERIES = false omits the small-x check: only for pairs known to have
// r2 >= r2_series, where the result is bitwise that of SERIES = true.
template <bool SERIES = true>
__device__ __forceinline__ void pair2(const ulonglong2 &hi, const ulonglong2 &lo, f32x2 g2,
                                      f32x2 txh, f32x2 tyh, f32x2 txl, f32x2 tyl,
                                      const GaussParams2 &gp, f32x2 &nx, f32x2 &ny) {
    const f32x2 dx = add2(sub2(txh, hi.x), sub2(txl, lo.x));
    const f32x2 dy = add2(sub2(tyh, hi.y), sub2(tyl, lo.y));
    const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, gp.eps));
    float ta, tb, ra, rb;
    unpack2(mul2(r2, gp.c_t), ta, tb);
    f32x2 om = sub2(gp.one, pack2(ex2_approx(ta), ex2_approx(tb)));
    unpack2(r2, ra, rb);
    if (SERIES && fminf(ra, rb) < gp.r2_series) {  // 1 - exp(-x) cancels: series
        float oa, ob;
        unpack2(om, oa, ob);
        if (ra < gp.r2_series) oa = series_om(ra, gp.c_x1);
        if (rb < gp.r2_series) ob = series_om(rb, gp.c_x1);
        om = pack2(oa, ob);
    }
    const f32x2 s = mul2(mul2(g2, om), pack2(rcp_approx(ra), rcp_approx(rb)));
    nx = fma2(dy, s, nx);
    ny = fma2(dx, s, ny);
}

// pair2_far on coordinates relative to a nearby centre c, one float each
// (x - c rounded once): for far pairs the rounding of the relative
// coordinates (|x - c| 2^-24, with |x - c| a few pair distances) stays near
// 1e-7 of the pair distance, so the hi/lo split is not needed there.
// loc = {x, x, y, y} of the source, txc/tyc the targets' relative coordinates.
__device__ __forceinline__ void pair2_far_local(const ulonglong2 &loc, f32x2 g2, f32x2 txc,
                                                f32x2 tyc, const GaussParams2 &gp, f32x2 &nx,
                                                f32x2 &ny) {
    const f32x2 dx = sub2(txc, loc.x);
    const f32x2 dy = sub2(tyc, loc.y);
    const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, gp.eps));
    float ra, rb;
    unpack2(r2, ra, rb);
    const f32x2 s = mul2(g2, pack2(rcp_approx(ra), rcp_approx(rb)));
    nx = fma2(dy, s, nx);
    ny = fma2(dx, s, ny);
}

// pair2 for pairs known to have r2 * log2(e)/ksigmasqr >= Y_FAR (see the file
// comment): om is 1.0f there and g * 1.0f = g, so this is bitwise pair2
// without the ex2.
__device__ __forceinline__ void pair2_far(const ulonglong2 &hi, const ulonglong2 &lo, f32x2 g2,
                                          f32x2 txh, f32x2 tyh, f32x2 txl, f32x2 tyl,
                                          const GaussParams2 &gp, f32x2 &nx, f32x2 &ny) {
    const f32x2 dx = add2(sub2(txh, hi.x), sub2(txl, lo.x));
    const f32x2 dy = add2(sub2(tyh, hi.y), sub2(tyl, lo.y));
    const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, gp.eps));
    float ra, rb;
    unpack2(r2, ra, rb);
    const f32x2 s = mul2(g2, pack2(rcp_approx(ra), rcp_approx(rb)));
    nx = fma2(dy, s, nx);
    ny = fma2(dx, s, ny);
}

// Cutoff (Rosenhead-Krasny) kernel of the reference's vv2par
// (src/cpp/blobs/c/vv2par_C/vv2par_C_cpu.c:143-148): s = g / (r^2 + sigma^2),
// nx += dy*s, ny += dx*s; s2 = {sigma^2, sigma^2}.  The pair2_far arithmetic
// with sigma^2 in place of 1e-12.
__device__ __forceinline__ void pair2_cutoff(const ulonglong2 &hi, const ulonglong2 &lo, f32x2 g2,
                                             f32x2 txh, f32x2 tyh, f32x2 txl, f32x2 tyl, f32x2 s2,
                                             f32x2 &nx, f32x2 &ny) {
    const f32x2 dx = add2(sub2(txh, hi.x), sub2(txl, lo.x));
    const f32x2 dy = add2(sub2(tyh, hi.y), sub2(tyl, lo.y));
    const f32x2 r2 = fma2(dx, dx, fma2(dy, dy, s2));
    float ra, rb;
    unpack2(r2, ra, rb);
    const f32x2 s = mul2(g2, pack2(rcp_approx(ra), rcp_approx(rb)));
    nx = fma2(dy, s, nx);
    ny = fma2(dx, s, ny);
}

}  // namespace pfd
