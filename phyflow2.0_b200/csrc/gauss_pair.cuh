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
#pragma once
#include "pf_common.cuh"

namespace pfd {

constexpr float X_SERIES = 0.25f;
constexpr float LOG2E_F = 1.4426950408889634f;

struct GaussParams {
    float c_t;       // -log2(e)/ksigmasqr  (argument of ex2)
    float c_x;       // 1/ksigmasqr
    float r2_series; // X_SERIES * ksigmasqr
};

__host__ __device__ inline GaussParams make_gauss_params(double ksigmasqr) {
    GaussParams p;
    p.c_t = (float)(-1.4426950408889634 / ksigmasqr);
    p.c_x = (float)(1.0 / ksigmasqr);
    p.r2_series = (float)(0.25 * ksigmasqr);
    return p;
}

// (1 - exp(-x)) / r2 * g given r2, with the series branch for small x.
__device__ __forceinline__ float gauss_s(float r2, float g, const GaussParams &p) {
    float e = ex2_approx(r2 * p.c_t);
    float om = 1.0f - e;
    if (r2 < p.r2_series) {
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

}  // namespace pfd
