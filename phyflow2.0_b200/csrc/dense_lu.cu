// dense_lu.cu -- LU factorisation with partial pivoting and the matching
// solve, FP64, for the panel system A gamma = RHS.
//
// The reference factorises the panel influence matrix once per geometry with
// scipy.linalg.lu_factor and solves every step with lu_solve
// (src/python/panels/__panelsClass.py:782, :960-962).  Here the matrix stays
// on the device: blocked right-looking LU (LAPACK getrf order of operations
// within a panel of LU_NB columns): per panel, one CTA factorises the
// LU_NB columns with row pivoting (ties to the smallest row), the rows of U to
// the right are solved against the unit lower block, and a tiled FP64 update
// subtracts L21 U12 from the trailing matrix.  Row-major storage; ipiv[k] is
// the row exchanged with row k at step k.  No device-side waits between
// CTAs: each phase is its own launch.
#include "pf_common.cuh"

#include <algorithm>

namespace {

constexpr int LU_NB = 32;         // panel width
constexpr int LU_THREADS = 256;   // panel / solve CTA
constexpr int GT = 64;            // trailing-update tile (GT x GT), 16 x 16 threads, 4 x 4 each

// Factorise columns [j0, j0+nb) of the row-major m x m matrix: pivot, swap
// whole rows, scale the column below the diagonal, update the panel.
__global__ void __launch_bounds__(LU_THREADS)
k_lu_panel(int64_t m, int j0, int nb, double *__restrict__ A, int32_t *__restrict__ ipiv,
           int32_t *__restrict__ info) {
    __shared__ double s_v[LU_THREADS];
    __shared__ int s_i[LU_THREADS];
    for (int k = j0; k < j0 + nb; ++k) {
        // pivot: max |A[r][k]| over r >= k, smallest r on ties
        double best = -1.0;
        int bi = k;
        for (int64_t r = k + threadIdx.x; r < m; r += LU_THREADS) {
            const double v = fabs(A[r * m + k]);
            if (v > best) {
                best = v;
                bi = (int)r;
            }
        }
        s_v[threadIdx.x] = best;
        s_i[threadIdx.x] = bi;
        __syncthreads();
        for (int s = LU_THREADS / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                const double a = s_v[threadIdx.x], b = s_v[threadIdx.x + s];
                const int ia = s_i[threadIdx.x], ib = s_i[threadIdx.x + s];
                if (b > a || (b == a && ib < ia)) {
                    s_v[threadIdx.x] = b;
                    s_i[threadIdx.x] = ib;
                }
            }
            __syncthreads();
        }
        const int p = s_i[0];
        if (threadIdx.x == 0) {
            ipiv[k] = p;
            if (A[(int64_t)p * m + k] == 0.0 && *info == 0) *info = k + 1;
        }
        if (p != k)
            for (int64_t c = threadIdx.x; c < m; c += LU_THREADS) {
                const double t = A[(int64_t)k * m + c];
                A[(int64_t)k * m + c] = A[(int64_t)p * m + c];
                A[(int64_t)p * m + c] = t;
            }
        __syncthreads();
        const double d = A[(int64_t)k * m + k];
        if (d != 0.0)
            for (int64_t r = k + 1 + threadIdx.x; r < m; r += LU_THREADS) A[r * m + k] /= d;
        __syncthreads();
        // rank-1 update of the remaining panel columns
        const int nc = j0 + nb - (k + 1);
        if (nc > 0)
            for (int64_t e = threadIdx.x; e < (m - k - 1) * nc; e += LU_THREADS) {
                const int64_t r = k + 1 + e / nc;
                const int c = k + 1 + (int)(e % nc);
                A[r * m + c] -= A[r * m + k] * A[(int64_t)k * m + c];
            }
        __syncthreads();
    }
}

// U12: rows [j0, j0+nb), columns c >= j0+nb, forward substitution with the
// unit lower nb x nb block (one thread per column).
__global__ void __launch_bounds__(LU_THREADS)
k_lu_trsm(int64_t m, int j0, int nb, double *__restrict__ A) {
    const int64_t c = (int64_t)j0 + nb + (int64_t)blockIdx.x * LU_THREADS + threadIdx.x;
    if (c >= m) return;
    for (int i = 1; i < nb; ++i) {
        double s = A[(int64_t)(j0 + i) * m + c];
        for (int k = 0; k < i; ++k)
            s -= A[(int64_t)(j0 + i) * m + j0 + k] * A[(int64_t)(j0 + k) * m + c];
        A[(int64_t)(j0 + i) * m + c] = s;
    }
}

// A22 -= L21 U12 over rows/columns >= j1 = j0 + nb, inner dimension nb.
__global__ void __launch_bounds__(256)
k_lu_update(int64_t m, int j0, int nb, double *__restrict__ A) {
    __shared__ double s_l[GT][LU_NB + 1];
    __shared__ double s_u[LU_NB][GT + 1];
    const int64_t j1 = (int64_t)j0 + nb;
    const int64_t r0 = j1 + (int64_t)blockIdx.y * GT, c0 = j1 + (int64_t)blockIdx.x * GT;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    for (int e = threadIdx.x; e < GT * LU_NB; e += 256) {
        const int r = e / LU_NB, k = e % LU_NB;
        s_l[r][k] = (r0 + r < m && k < nb) ? A[(r0 + r) * m + j0 + k] : 0.0;
        const int k2 = e / GT, c = e % GT;
        s_u[k2][c] = (c0 + c < m && k2 < nb) ? A[(int64_t)(j0 + k2) * m + c0 + c] : 0.0;
    }
    __syncthreads();
    double acc[4][4] = {};
    for (int k = 0; k < nb; ++k) {
        double l[4], u[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            l[a] = s_l[ty + 16 * a][k];
            u[a] = s_u[k][tx + 16 * a];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = fma(l[a], u[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int64_t r = r0 + ty + 16 * a, c = c0 + tx + 16 * b;
            if (r < m && c < m) A[r * m + c] -= acc[a][b];
        }
}

// x = A^-1 b from the factors: row exchanges, unit-lower forward and upper
// back substitution, one CTA, column-oriented updates.
__global__ void __launch_bounds__(LU_THREADS)
k_lu_solve(int64_t m, const double *__restrict__ LU, const int32_t *__restrict__ ipiv,
           double *__restrict__ b) {
    if (threadIdx.x == 0)
        for (int64_t k = 0; k < m; ++k) {
            const int p = ipiv[k];
            if (p != k) {
                const double t = b[k];
                b[k] = b[p];
                b[p] = t;
            }
        }
    __syncthreads();
    for (int64_t k = 0; k < m; ++k) {
        const double bk = b[k];
        for (int64_t r = k + 1 + threadIdx.x; r < m; r += LU_THREADS) b[r] -= LU[r * m + k] * bk;
        __syncthreads();
    }
    for (int64_t k = m - 1; k >= 0; --k) {
        if (threadIdx.x == 0) b[k] /= LU[k * m + k];
        __syncthreads();
        const double bk = b[k];
        for (int64_t r = threadIdx.x; r < k; r += LU_THREADS) b[r] -= LU[r * m + k] * bk;
        __syncthreads();
    }
}

}  // namespace

extern "C" pf_status pf_dense_lu_factor(pf_ctx *ctx, int64_t m, double *a, int32_t *ipiv,
                                        int32_t *info_dev, void *stream) {
    PF_RANGE("pf_dense_lu_factor");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_dense_lu_factor: NULL context");
    PF_CHECK_ARG(m >= 0 && m <= 32768, "pf_dense_lu_factor: m = %lld outside [0, 32768]",
                 (long long)m);
    PF_CHECK_ARG(m == 0 || (a && ipiv && info_dev), "pf_dense_lu_factor: NULL array");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (m == 0) return PF_OK;
    PF_CUDA_TRY(cudaMemsetAsync(info_dev, 0, sizeof(int32_t), st));
    for (int64_t j0 = 0; j0 < m; j0 += LU_NB) {
        const int nb = (int)std::min<int64_t>(LU_NB, m - j0);
        k_lu_panel<<<1, LU_THREADS, 0, st>>>(m, (int)j0, nb, a, ipiv, info_dev);
        PF_TRY(pf::launch_status("k_lu_panel"));
        const int64_t rest = m - j0 - nb;
        if (rest <= 0) continue;
        k_lu_trsm<<<(unsigned)pf::ceil_div(rest, LU_THREADS), LU_THREADS, 0, st>>>(m, (int)j0, nb,
                                                                                  a);
        PF_TRY(pf::launch_status("k_lu_trsm"));
        const unsigned gt = (unsigned)pf::ceil_div(rest, GT);
        k_lu_update<<<dim3(gt, gt), 256, 0, st>>>(m, (int)j0, nb, a);
        PF_TRY(pf::launch_status("k_lu_update"));
    }
    return PF_OK;
}

extern "C" pf_status pf_dense_lu_solve(pf_ctx *ctx, int64_t m, const double *lu,
                                       const int32_t *ipiv, double *b, void *stream) {
    PF_RANGE("pf_dense_lu_solve");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_dense_lu_solve: NULL context");
    PF_CHECK_ARG(m >= 0 && m <= 32768, "pf_dense_lu_solve: m = %lld outside [0, 32768]",
                 (long long)m);
    PF_CHECK_ARG(m == 0 || (lu && ipiv && b), "pf_dense_lu_solve: NULL array");
    pf::DeviceGuard dg(ctx->device);
    if (m == 0) return PF_OK;
    k_lu_solve<<<1, LU_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(m, lu, ipiv, b);
    return pf::launch_status("k_lu_solve");
}
