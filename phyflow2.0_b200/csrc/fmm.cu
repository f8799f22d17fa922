// fmm.cu -- 2D fast multipole method for Gaussian vortex blobs on B200.
//
// Tree: uniform quadtree over the bounding square of sources and targets,
// every level a dense 2^l x 2^l grid addressed by Morton index (box (l, m) at
// global slot off[l] + m, off[l] = (4^l - 1)/3).  Particles are counting-
// sorted by leaf Morton key (ties in input order, so every sum has a fixed
// order) -- this replaces the reference's median-split partition
// (src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmmsort.cpp:441-790).
//
// Expansions (FP64, complex, scaled by the box width w so that all
// coefficients are O(sum |g|)):
//   multipole  M(z) = sum_j g_j / (z - z_j) = sum_k a_k w^k / (z - c)^(k+1),
//              a_k = sum_j g_j ((z_j - c)/w)^k                       (P2M)
//   local      L(z) = (1/w) sum_n lam_n ((z - c)/w)^n
//   M2M  a'_k  = sum_{m<=k} C(k,m) tau^(k-m) 2^-m a_m,  tau = (c_child - c_par)/w_par
//   M2L  lam_n += sum_k (-1)^(k+1) C(n+k,k) rho^(n+k+1) a_k,  rho = 1/(i + i j)
//              for a far box at integer offset (i, j): the operator depends
//              only on the offset, so rho^m is tabulated per offset
//   L2L  lam'_n = (1/2) sum_{m>=n} C(m,n) tau^(m-n) 2^-n lam_m
//   L2P  W = L(z);  u = Im W / 2pi,  v = Re W / 2pi
// (reference counterparts: mpexp_init fmm.cpp:1452-1509, shift_m2m
// fmmshift.cpp:80-236, shift_m2ps fmmshift.cpp:237-621, shift_p2p
// fmmshift.cpp:622-767, mpexp_eval fmm.cpp:1875-1931).
// M2M, M2L and L2L run on the FP64 tensor cores (mma.sync m8n8k4 .f64):
// their operators are fixed matrices (per child position, or the binomial
// matrix between the scalings by rho), applied to four boxes per warp task.
//
// Near field: the Gaussian kernel itself, FP32 with hi/lo coordinates and
// compensated accumulation (gauss_pair.cuh), for every target of a P2P block
// (2^kb x 2^kb leaves) against the block's source leaves; those leaves are
// sorted by Morton index and merged into runs of consecutive leaves, which
// are contiguous in the sorted particle arrays, and streamed through shared
// memory in full tiles.  The interaction lists come from fmm_plan.cu.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "fmm_api.cuh"
#include "fmm_plan.cuh"
#include "gauss_pair.cuh"
#include "scan.cuh"
#include "segsort.cuh"

#include "direct_api.cuh"

namespace {

using pf::fmmx::P2PDesc;
using pf::fmmx::P2PWork;

constexpr double THETA = 0.5;
constexpr double INV_2PI = 0.15915494309189535;
constexpr int MAX_LEVEL = pf::fmmx::MAX_LEVEL;
constexpr int P2P_SETUP_THREADS = 128;
constexpr int P2P_QMAX = 1024;   // source leaves per P2P block
constexpr int P2P_RUNS_SM = 64;  // runs staged in shared memory at a time
constexpr int P2P_BUF = 64;      // sources per warp buffer (three buffers)
// unroll of the pair loop over a full chunk: the kernel holds nine copies of
// it (targets per lane x mode), which must stay within the instruction cache
constexpr int P2P_UNROLL = 8;
constexpr int P2P_MIN_CTAS = 20; // one-warp CTAs resident per SM: 96 registers each
constexpr unsigned INVALID_KEY = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// Morton helpers (x in even bits, y in odd bits)
__host__ __device__ __forceinline__ uint32_t part1by1(uint32_t v) {
    v &= 0x0000ffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
__host__ __device__ __forceinline__ uint32_t compact1by1(uint32_t v) {
    v &= 0x55555555u;
    v = (v | (v >> 1)) & 0x33333333u;
    v = (v | (v >> 2)) & 0x0f0f0f0fu;
    v = (v | (v >> 4)) & 0x00ff00ffu;
    v = (v | (v >> 8)) & 0x0000ffffu;
    return v;
}
__host__ __device__ __forceinline__ uint32_t morton2(uint32_t x, uint32_t y) {
    return part1by1(x) | (part1by1(y) << 1);
}

// Morton code of (x + dx, y + dy) from the code m of (x, y) and the dilated
// offset d = morton2(dx mod 2^16, dy mod 2^16): each coordinate's bits are
// added with the other coordinate's bit positions filled with ones, so the
// carries run through them ("dilated integer" addition).  Exact whenever the
// shifted coordinates lie in [0, 2^16).
__device__ __forceinline__ uint32_t morton_add(uint32_t m, uint32_t d) {
    const uint32_t xm = 0x55555555u, ym = 0xaaaaaaaau;
    return (((m | ym) + (d & xm)) & xm) | (((m | xm) + (d & ym)) & ym);
}

// leaf coordinate of a position: floor((x - x0) / w) clamped to [0, 2^L)
__device__ __forceinline__ uint32_t leaf_coord(double x, double x0, double w, int L) {
    const double q = floor(__ddiv_rn(__dsub_rn(x, x0), w));
    const double hi = (double)((1u << L) - 1u);
    return (uint32_t)fmin(fmax(q, 0.0), hi);
}

// ---------------------------------------------------------------------------
// bounding box with order-preserving integer images of doubles
__device__ __forceinline__ unsigned long long ord_d(double v) {
    unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ inline double unord_d(unsigned long long u) {
    u = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
    double d;
    memcpy(&d, &u, 8);
    return d;
}

struct BBox {
    unsigned long long mnx, mxx, mny, mxy;
    int bad;
    int pad[7];
};

__global__ void k_bbox_init(BBox *b) {
    b->mnx = b->mny = ~0ull;
    b->mxx = b->mxy = 0ull;
    b->bad = 0;
}

__global__ void __launch_bounds__(256)
k_bbox(const double *__restrict__ x, const double *__restrict__ y, int64_t n, BBox *b) {
    unsigned long long mnx = ~0ull, mxx = 0, mny = ~0ull, mxy = 0;
    int bad = 0;
    // four independent loads of x and y per thread in flight
    const int64_t stride = (int64_t)gridDim.x * 256;
    for (int64_t i0 = (int64_t)blockIdx.x * 256 + threadIdx.x; i0 < n; i0 += 4 * stride) {
        double a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = i0 + u * stride;
            a[u] = i < n ? x[i] : 0.0;
            c[u] = i < n ? y[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u * stride >= n) continue;
            if (!isfinite(a[u]) || !isfinite(c[u])) {
                bad = 1;
                continue;
            }
            const unsigned long long oa = ord_d(a[u]), oc = ord_d(c[u]);
            mnx = min(mnx, oa);
            mxx = max(mxx, oa);
            mny = min(mny, oc);
            mxy = max(mxy, oc);
        }
    }
    for (int o = 16; o; o >>= 1) {
        mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    // block reduction, then one set of atomics per block
    __shared__ unsigned long long s_v[4][8];
    __shared__ int s_bad[8];
    const int wid = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_v[0][wid] = mnx;
        s_v[1][wid] = mxx;
        s_v[2][wid] = mny;
        s_v[3][wid] = mxy;
        s_bad[wid] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) {
            mnx = min(mnx, s_v[0][w]);
            mxx = max(mxx, s_v[1][w]);
            mny = min(mny, s_v[2][w]);
            mxy = max(mxy, s_v[3][w]);
            bad |= s_bad[w];
        }
        atomicMin(&b->mnx, mnx);
        atomicMax(&b->mxx, mxx);
        atomicMin(&b->mny, mny);
        atomicMax(&b->mxy, mxy);
        if (bad) atomicOr(&b->bad, 1);
    }
}

// ---------------------------------------------------------------------------
// counting sort by leaf key
__global__ void __launch_bounds__(256)
k_leaf_keys(const double *__restrict__ x, const double *__restrict__ y, int64_t n, double x0,
            double y0, double wl, int L, uint32_t *__restrict__ key, int32_t *__restrict__ rank,
            int32_t *__restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = morton2(leaf_coord(x[i], x0, wl, L), leaf_coord(y[i], y0, wl, L));
    key[i] = k;
    if (rank) rank[i] = atomicAdd(&cnt[k], 1);
}

__global__ void __launch_bounds__(256)
k_place(int64_t n, const uint32_t *__restrict__ key, const int32_t *__restrict__ rank,
        const int32_t *__restrict__ start, int32_t *__restrict__ perm, int32_t *__restrict__ big,
        int32_t *__restrict__ big_n) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const int64_t p = (int64_t)start[key[i]] + rank[i];
    if (PF_IDX_OK(p, n, 201)) perm[p] = (int32_t)i;
    // a leaf of more than SEG_SMALL particles (exactly one has this rank) is
    // listed for the segment sort
    if (rank[i] == pf::SEG_SMALL) big[atomicAdd(big_n, 1)] = (int32_t)key[i];
}

__host__ __device__ __forceinline__ int64_t level_off(int l) {
    return ((((int64_t)1) << (2 * l)) - 1) / 3;
}

// Sorted copies of the points in leaf order, each leaf's particles by input
// index (the counting sort's atomic ranks are not reproducible; this fixes
// every later sum's order).  Thread j takes the particle i = perm[j] that the
// counting sort placed in its leaf's range [s0, s0 + c); its final position
// is s0 + (number of the leaf's particles with a smaller index), found by
// reading the leaf's c entries of perm (leaves above SEG_SMALL particles are
// already in index order: seg_sort_listed).  Writes the final permutation to
// perm_out and, at that position, FP64 x, y (g), the hi/lo float4 and float g
// of the near field and the leaf key.
__global__ void __launch_bounds__(256)
k_gather_sorted(int64_t n, const int32_t *__restrict__ perm, const uint32_t *__restrict__ key,
                const int32_t *__restrict__ start, const int32_t *__restrict__ cnt,
                const double *__restrict__ x, const double *__restrict__ y,
                const double *__restrict__ g, int32_t *__restrict__ perm_out,
                double *__restrict__ sx, double *__restrict__ sy, double *__restrict__ sg,
                float4 *__restrict__ hl, float *__restrict__ g32, uint32_t *__restrict__ skey) {
    const int64_t j = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (j >= n) return;
    const int32_t i = perm[j];
    if (!PF_IDX_OK(i, n, 202)) return;
    const uint32_t m = key[i];
    const double a = x[i], b = y[i];
    const double gi = g ? g[i] : 0.0;
    const int s0 = start[m], c = cnt[m];
    int64_t d = j;
    if (c <= pf::SEG_SMALL && PF_IDX_OK((int64_t)s0 + c - 1, n, 206)) {
        int r = 0;
        for (int q = 0; q < c; ++q) r += perm[s0 + q] < i;
        d = (int64_t)s0 + r;
    }
    perm_out[d] = i;
    if (skey) skey[d] = m;  // leaf key in sorted order (targets)
    sx[d] = a;
    sy[d] = b;
    float4 h;
    pfd::split_hilo(a, h.x, h.z);
    pfd::split_hilo(b, h.y, h.w);
    hl[d] = h;
    if (g) {
        sg[d] = gi;
        g32[d] = (float)gi;
    }
}

// Box counts of nlev (<= 4) coarser levels from level lc: CTA b owns the
// 4^nlev level-lc boxes below box b of level lc - nlev (one contiguous Morton
// range) and sums them up level by level in shared memory (integer sums:
// exact, any order).
__global__ void __launch_bounds__(256)
k_count_up(int lc, int nlev, int32_t *__restrict__ cnt_all) {
    __shared__ int32_t s_c[256];
    const int nch = 1 << (2 * nlev);
    if ((int)threadIdx.x < nch)
        s_c[threadIdx.x] = cnt_all[level_off(lc) + (int64_t)blockIdx.x * nch + threadIdx.x];
    __syncthreads();
    for (int j = 1; j <= nlev; ++j) {
        const int np = nch >> (2 * j);
        int32_t v = 0;
        if ((int)threadIdx.x < np)
            v = s_c[4 * threadIdx.x] + s_c[4 * threadIdx.x + 1] + s_c[4 * threadIdx.x + 2] +
                s_c[4 * threadIdx.x + 3];
        __syncthreads();
        if ((int)threadIdx.x < np) {
            s_c[threadIdx.x] = v;
            cnt_all[level_off(lc - j) + (int64_t)blockIdx.x * np + threadIdx.x] = v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// complex helpers
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // a*b + c
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

// P2M: one thread per leaf
template <int NP>
__global__ void __launch_bounds__(128)
k_p2m(int L, double x0, double y0, double wl, const int32_t *__restrict__ start,
      const int32_t *__restrict__ cnt, const double *__restrict__ sx,
      const double *__restrict__ sy, const double *__restrict__ sg, double2 *__restrict__ M) {
    // four consecutive lanes per leaf, lane q taking the leaf's particles
    // q, q + 4, ...; the four partial expansions are added in a fixed tree order
    const int64_t nleaf = (int64_t)1 << (2 * L);
    const int64_t t = (int64_t)blockIdx.x * 128 + threadIdx.x;
    const int64_t m = t >> 2;
    const int q = (int)(t & 3);
    const bool live = m < nleaf;
    const int c = live ? cnt[m] : 0;
    const uint32_t ix = compact1by1((uint32_t)m), iy = compact1by1((uint32_t)m >> 1);
    const double cx = x0 + ((double)ix + 0.5) * wl, cy = y0 + ((double)iy + 0.5) * wl;
    const double iw = 1.0 / wl;
    double2 a[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) a[k] = make_double2(0.0, 0.0);
    const int s0 = live ? start[m] : 0;
    for (int j = q; j < c; j += 4) {
        const double2 z = make_double2((sx[s0 + j] - cx) * iw, (sy[s0 + j] - cy) * iw);
        double2 zk = make_double2(sg[s0 + j], 0.0);
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            a[k].x += zk.x;
            a[k].y += zk.y;
            zk = cmul(zk, z);
        }
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) {
#pragma unroll
        for (int o = 1; o <= 2; o <<= 1) {
            a[k].x += __shfl_xor_sync(0xffffffffu, a[k].x, o);
            a[k].y += __shfl_xor_sync(0xffffffffu, a[k].y, o);
        }
    }
    if (!live || c == 0) return;
    const int64_t base = ((((int64_t)1 << (2 * L)) - 1) / 3 + m) * NP;
#pragma unroll
    for (int k = 0; k < NP; ++k)
        if ((k & 3) == q) M[base + k] = a[k];
}


// One FP64 tensor-core product d = a b + d of an 8 x 4 by 4 x 8 tile
// (mma.sync m8n8k4 .f64; tcgen05 has no FP64 kind).  Fragments: a = A[lane/4]
// [lane%4], b = B[lane%4][lane/4], (d0, d1) = D[lane/4][2 (lane%4) + 0, 1].
__device__ __forceinline__ void mma_f64(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// M2M and L2L on the FP64 tensor cores.  The translation of a box's
// expansion to (M2M) or from (L2L) child position c is a fixed complex NP x NP
// matrix T_c (lower triangular for M2M, upper for L2L).  A warp task applies
// it to four boxes at once: the B operand holds their coefficients (column
// 2j real, 2j + 1 imaginary parts of box j), the A operand the real and the
// imaginary part of T_c, from fragment tables built with the plan
// (frag[c][part][mt][ks][lane] = part of T_c[8 mt + lane/4][4 ks + lane%4]);
// tiles of zeros are skipped.  With U = Re T B and V = Im T B, lane (box
// lane%4, row n = lane/4 + 8 mt) holds Re = U_re - V_im and Im = U_im + V_re.
template <int NP>
struct TcShape {
    static constexpr int MT = (NP + 7) / 8, KS = (NP + 3) / 4;
};

// TRI = 1: T[row][col] = 0 for col > row (M2M); TRI = -1: for col < row (L2L)
template <int TRI>
__device__ __forceinline__ constexpr bool tc_tile_live(int mt, int ks) {
    return TRI > 0 ? 4 * ks <= 8 * mt + 7 : 4 * ks + 3 >= 8 * mt;
}

// d[mt] = T_c b for the lane's (box lane%4, rows lane/4 + 8 mt); b[s] = the
// lane's B element of k block s (row 4 s + lane%4, column lane/4).
template <int NP, int TRI>
__device__ __forceinline__ void tc_apply(const double *__restrict__ fr,
                                         const double (&b)[TcShape<NP>::KS],
                                         double2 (&d)[TcShape<NP>::MT]) {
    constexpr int MT = TcShape<NP>::MT, KS = TcShape<NP>::KS;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
        double u0 = 0.0, u1 = 0.0, v0 = 0.0, v1 = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            if (!tc_tile_live<TRI>(mt, ks)) continue;
            mma_f64(u0, u1, __ldg(fr + ((0 * MT + mt) * KS + ks) * 32 + lane), b[ks]);
            mma_f64(v0, v1, __ldg(fr + ((1 * MT + mt) * KS + ks) * 32 + lane), b[ks]);
        }
        d[mt] = make_double2(u0 - v1, u1 + v0);
    }
}

// The lane's B elements of four boxes' coefficients: coef(j, m) is
// coefficient m of box j (zero for an empty box).
template <int NP, class Coef>
__device__ __forceinline__ void tc_load_b(Coef coef, double (&b)[TcShape<NP>::KS]) {
    const int lane = threadIdx.x & 31;
    const int j = lane >> 3, part = (lane >> 2) & 1, kq = lane & 3;
#pragma unroll
    for (int ks = 0; ks < TcShape<NP>::KS; ++ks) {
        const int m = 4 * ks + kq;
        const double2 v = m < NP ? coef(j, m) : make_double2(0.0, 0.0);
        b[ks] = part ? v.y : v.x;
    }
}

constexpr int TC_THREADS = 128;  // four warp tasks per CTA

// M2M into parent level l for four consecutive parents per warp task:
// out_j[k] = sum_c T_c (children 4 P_j + c, empty ones as zeros), written for
// the non-empty parents.  With two_level, the same warp then forms the
// grandparent (level l - 1, box task) from those four parents.
template <int NP>
__global__ void __launch_bounds__(TC_THREADS)
k_m2m_tc(int l, bool two_level, const int32_t *__restrict__ scnt, double2 *__restrict__ M,
         const double *__restrict__ frag /* [4][2][MT][KS][32] */) {
    constexpr int MT = TcShape<NP>::MT;
    constexpr int FR = 2 * MT * TcShape<NP>::KS * 32;  // doubles per child position
    __shared__ double2 s_par[TC_THREADS / 32][4][NP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t task = (int64_t)blockIdx.x * (TC_THREADS / 32) + wid;
    if (task >= ((int64_t)1 << (2 * l)) / 4) return;  // the whole warp
    const int64_t p0 = level_off(l) + 4 * task;        // parents p0 .. p0 + 3
    const int64_t c0 = level_off(l + 1) + 16 * task;   // their children
    double2 out[MT];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) out[mt] = make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double b[TcShape<NP>::KS];
        tc_load_b<NP>(
            [&](int j, int m) {
                const int64_t ch = c0 + 4 * j + c;
                const double2 v = M[ch * NP + m];  // loaded with the count
                return scnt[ch] != 0 ? v : make_double2(0.0, 0.0);
            },
            b);
        double2 d[MT];
        tc_apply<NP, 1>(frag + c * FR, b, d);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
            out[mt] = make_double2(out[mt].x + d[mt].x, out[mt].y + d[mt].y);
    }
    const int jd = lane & 3, nr = lane >> 2;
    const bool live = scnt[p0 + jd] != 0;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
        const int n = 8 * mt + nr;
        if (n >= NP) continue;
        if (live) M[(p0 + jd) * NP + n] = out[mt];
        s_par[wid][jd][n] = live ? out[mt] : make_double2(0.0, 0.0);
    }
    if (!two_level) return;
    __syncwarp();
    // grandparent (task) of level l - 1 from the four parents: column 0 only
    double2 g[MT];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) g[mt] = make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double b[TcShape<NP>::KS];
        tc_load_b<NP>([&](int j, int m) { return j == 0 ? s_par[wid][c][m] : make_double2(0.0, 0.0); },
                      b);
        double2 d[MT];
        tc_apply<NP, 1>(frag + c * FR, b, d);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) g[mt] = make_double2(g[mt].x + d[mt].x, g[mt].y + d[mt].y);
    }
    const int64_t gp = level_off(l - 1) + task;
    if (jd == 0 && scnt[gp] != 0)
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int n = 8 * mt + nr;
            if (n < NP) M[gp * NP + n] = g[mt];
        }
}

// L2L from parent level l - 1 into child level l for four consecutive parents
// per warp task: child 4 P_j + c += T_c L_{P_j}, for the non-empty children.
// With two_level the same warp first forms the four parents themselves from
// their parent (level l - 2, box task), then their children.
template <int NP>
__global__ void __launch_bounds__(TC_THREADS)
k_l2l_tc(int l, bool two_level, const int32_t *__restrict__ tcnt, double2 *__restrict__ Lc,
         const double *__restrict__ frag /* [4][2][MT][KS][32] */) {
    constexpr int MT = TcShape<NP>::MT;
    constexpr int FR = 2 * MT * TcShape<NP>::KS * 32;
    __shared__ double2 s_par[TC_THREADS / 32][4][NP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int jd = lane & 3, nr = lane >> 2;
    const int64_t task = (int64_t)blockIdx.x * (TC_THREADS / 32) + wid;
    if (task >= ((int64_t)1 << (2 * l)) / 16) return;  // the whole warp
    const int64_t p0 = level_off(l - 1) + 4 * task;     // parents p0 .. p0 + 3
    const int64_t c0 = level_off(l) + 16 * task;        // their children
    if (two_level) {
        // the parents (children of box `task` of level l - 2): column 0 only
        const int64_t gp = level_off(l - 2) + task;
        const bool glive = tcnt[gp] != 0;
        double b[TcShape<NP>::KS];
        tc_load_b<NP>([&](int j, int m) {
            return (j == 0 && glive) ? Lc[gp * NP + m] : make_double2(0.0, 0.0);
        }, b);
        // lanes of column 0 (jd == 0) take parent c's rows: its own local
        // expansion is loaded before the products
        double2 old[4][MT];
        bool plive[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            plive[c] = tcnt[p0 + c] != 0;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const int n = 8 * mt + nr;
                old[c][mt] = (jd == 0 && n < NP) ? Lc[(p0 + c) * NP + n] : make_double2(0.0, 0.0);
            }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double2 d[MT];
            tc_apply<NP, -1>(frag + c * FR, b, d);
            if (jd == 0)
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    const int n = 8 * mt + nr;
                    if (n >= NP) continue;
                    double2 v = make_double2(0.0, 0.0);
                    if (plive[c]) {
                        v = make_double2(old[c][mt].x + d[mt].x, old[c][mt].y + d[mt].y);
                        Lc[(p0 + c) * NP + n] = v;
                    }
                    s_par[wid][c][n] = v;  // broadcast to the warp by shared memory
                }
        }
        __syncwarp();
    } else {
        for (int t = lane; t < 4 * NP; t += 32) {
            const int j = t / NP, n = t - j * NP;
            s_par[wid][j][n] = tcnt[p0 + j] != 0 ? Lc[(p0 + j) * NP + n] : make_double2(0.0, 0.0);
        }
        __syncwarp();
    }
    // the children's own local expansions, loaded before the products
    double2 old[4][MT];
    bool clive[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int64_t ch = c0 + 4 * jd + c;
        clive[c] = tcnt[ch] != 0;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int n = 8 * mt + nr;
            old[c][mt] = n < NP ? Lc[ch * NP + n] : make_double2(0.0, 0.0);
        }
    }
    double b[TcShape<NP>::KS];
    tc_load_b<NP>([&](int j, int m) { return s_par[wid][j][m]; }, b);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        double2 d[MT];
        tc_apply<NP, -1>(frag + c * FR, b, d);
        if (!clive[c]) continue;
        const int64_t ch = c0 + 4 * jd + c;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int n = 8 * mt + nr;
            if (n < NP)
                Lc[ch * NP + n] = make_double2(old[c][mt].x + d[mt].x, old[c][mt].y + d[mt].y);
        }
    }
}

constexpr int M2L_THREADS = 128;  // 4 warps, four target boxes each

// M2L for all levels 2..L on the FP64 tensor cores.  One translation adds
//   L_n += r^(n+1) sum_k C(n+k, k) c_k,   c_k = (-1)^(k+1) M_k r^k
// (r: the operator's powers), so the binomial matrix is the same for every
// translation.  A warp holds it as the A operand (rows n, columns k, in 8 x 4
// fragments) and takes four target boxes of one level with the same far list
// (same position class: Morton indices r0 + q stride) as the 8 columns of B,
// the real and imaginary parts of their c.  Per far-list entry: B from the
// four sources' multipoles, KS mma per 8 rows, then lane (n = lane/4 + 8 mt,
// box lane%4) scales its (re, im) pair by r^(n+1) into its coefficient.
template <int NP>
__global__ void __launch_bounds__(M2L_THREADS)
k_m2l(int L, int Bp, int64_t nquad, const int32_t *__restrict__ scnt,
      const int32_t *__restrict__ tcnt, const double2 *__restrict__ M, double2 *__restrict__ Lc,
      const int4 *__restrict__ far, const int32_t *__restrict__ far_ptr, int maxpos,
      const double2 *__restrict__ pw /* [nop][NP+1] */, const double *__restrict__ binom,
      unsigned long long *__restrict__ ntrans) {
    constexpr int MT = (NP + 7) / 8, KS = (NP + 3) / 4;
    const int lane = threadIdx.x & 31;
    const int64_t u = (int64_t)blockIdx.x * (M2L_THREADS / 32) + (threadIdx.x >> 5);
    if (u >= nquad) return;  // the whole warp
    int l = 2;
    int64_t j = u;
    while (l < L && j >= ((int64_t)1 << (2 * l)) / 4) {
        j -= ((int64_t)1 << (2 * l)) / 4;
        ++l;
    }
    const int64_t stride = (l == L) ? (int64_t)Bp * Bp : 4;
    const int64_t r0 = (j / stride) * 4 * stride + (j % stride);
    // B column lane/4: box tb, part (0 real, 1 imaginary); B row k = 4 s + kq
    const int tb = lane >> 3, part = (lane >> 2) & 1, kq = lane & 3;
    // D: box td, rows n = nr + 8 mt
    const int td = lane & 3, nr = lane >> 2;
    const uint32_t mb = (uint32_t)(r0 + tb * stride);
    const int64_t lo = level_off(l);
    const bool liveb = tcnt[lo + mb] != 0;
    if (!__any_sync(0xffffffffu, liveb)) return;
    const bool lived = __shfl_sync(0xffffffffu, liveb, 8 * td);
    double af[MT][KS];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            const int n = 8 * mt + nr, k = 4 * s + kq;
            af[mt][s] = (n < NP && k < NP) ? binom[k * NP + n] : 0.0;
        }
    const int ixb = (int)compact1by1(mb), iyb = (int)compact1by1(mb >> 1);
    // the same for the four boxes
    const int pos = (l == L) ? ((ixb % Bp) + Bp * (iyb % Bp)) : ((ixb & 1) | ((iyb & 1) << 1));
    const int side = 1 << l;
    const int e0 = far_ptr[l * maxpos + pos];
    const int len = far_ptr[l * maxpos + pos + 1] - e0;
    const double sgn = (kq & 1) ? 1.0 : -1.0;  // (-1)^(k+1)
    double2 acc[MT];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) acc[mt] = make_double2(0.0, 0.0);
    unsigned nt = 0;
    for (int e = 0; e < len; ++e) {
        const int4 f = far[e0 + e];
        const int sx = ixb + f.x, sy = iyb + f.y;
        const bool inr = liveb && sx >= 0 && sy >= 0 && sx < side && sy < side;
        const int64_t sg = inr ? lo + morton_add(mb, (uint32_t)f.w) : 0;
        // the source's count and multipole are loaded together (the box is
        // in range either way); an empty source is then skipped
        const int cs = inr ? scnt[sg] : 0;
        const double2 *rp = pw + (int64_t)f.z * (NP + 1);
        double2 mv[KS], rv[KS];
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            const int k = 4 * s + kq;
            mv[s] = (inr && k < NP) ? M[sg * NP + k] : make_double2(0.0, 0.0);
            rv[s] = (k < NP) ? rp[k] : make_double2(0.0, 0.0);
        }
        const bool use = inr && cs != 0;
        if (!__any_sync(0xffffffffu, use)) continue;
        const bool used = __shfl_sync(0xffffffffu, use, 8 * td);
        nt += ((lane & 7) == 0 && use) ? 1u : 0u;
        double b[KS];
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            const double2 m = mv[s], r = rv[s];
            const double v = part ? fma(m.x, r.y, m.y * r.x) : fma(m.x, r.x, -(m.y * r.y));
            b[s] = use ? sgn * v : 0.0;
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            double d0 = 0.0, d1 = 0.0;
#pragma unroll
            for (int s = 0; s < KS; ++s) mma_f64(d0, d1, af[mt][s], b[s]);
            const int n = 8 * mt + nr;
            if (used && n < NP) acc[mt] = cfma(rp[n + 1], make_double2(d0, d1), acc[mt]);
        }
    }
    if (lived) {
        const int64_t bgd = lo + r0 + td * stride;
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int n = 8 * mt + nr;
            if (n < NP) Lc[bgd * NP + n] = acc[mt];
        }
    }
    nt = __reduce_add_sync(0xffffffffu, nt);
    if (lane == 0 && nt) atomicAdd(ntrans, (unsigned long long)nt);
}

// ---------------------------------------------------------------------------
// P2P run lists (once per plan; geometry only).  For P2P block b, the source
// leaves b's origin + q are sorted by Morton index and merged into runs of
// consecutive indices; consecutive leaves are contiguous in the sorted
// particle arrays, so a run is one particle range.  Pass 1 (runs == nullptr)
// writes the run count of each block, pass 2 the runs (first, last leaf).
__global__ void __launch_bounds__(P2P_SETUP_THREADS)
k_p2p_runs(int L, int kb, const int2 *__restrict__ q, int nq, int nqp,
           int32_t *__restrict__ nruns_or_off, int2 *__restrict__ runs) {
    __shared__ uint32_t s_key[P2P_QMAX];
    __shared__ int s_n;
    const uint32_t b = blockIdx.x;
    const int ox = (int)(compact1by1(b) << kb), oy = (int)(compact1by1(b >> 1) << kb);
    const int side = 1 << L;
    for (int t = threadIdx.x; t < nqp; t += P2P_SETUP_THREADS) {
        uint32_t k = INVALID_KEY;
        if (t < nq) {
            const int lx = ox + q[t].x, ly = oy + q[t].y;
            if (lx >= 0 && ly >= 0 && lx < side && ly < side) k = morton2(lx, ly);
        }
        s_key[t] = k;
    }
    __syncthreads();
    for (int kk = 2; kk <= nqp; kk <<= 1) {
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < nqp; t += P2P_SETUP_THREADS) {
                const int p = t ^ j;
                if (p > t) {
                    const uint32_t a = s_key[t], c = s_key[p];
                    const bool up = ((t & kk) == 0);
                    if ((a > c) == up) {
                        s_key[t] = c;
                        s_key[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int nr = 0;
        const int base_out = runs ? nruns_or_off[b] : 0;
        for (int base = 0; base < nqp; base += 32) {
            const int t = base + lane;
            const uint32_t k = (t < nqp) ? s_key[t] : INVALID_KEY;
            const bool valid = k != INVALID_KEY;
            const bool head = valid && (t == 0 || s_key[t - 1] + 1u != k);
            const uint32_t kn = (t + 1 < nqp) ? s_key[t + 1] : INVALID_KEY;
            const bool tail = valid && (kn == INVALID_KEY || kn != k + 1u);
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (runs) {
                if (head) runs[base_out + nr + __popc(hm & ((1u << lane) - 1u))].x = (int)k;
                // the run index of a tail is the number of heads at or before it, minus one
                if (tail) runs[base_out + nr + __popc(hm & ((2u << lane) - 1u)) - 1].y = (int)k;
            }
            nr += __popc(hm);
        }
        if (lane == 0) s_n = nr;
    }
    __syncthreads();
    if (!runs && threadIdx.x == 0) nruns_or_off[b] = s_n;
}

// P2P near field: one warp (one CTA) per P2P block, its targets in balanced
// groups of at most 96.  Targets a and b of a lane run packed (f32x2); in a
// group of 65..96 the remaining targets are spread over the warp, each lane
// taking a share of the sources (p2p_split_sums).  Pair code modes, chosen
// per source from its box distance to the group's target box (with a
// rounding margin):
//   P2P_FAR:    sources beyond sqrt(r2_far): no ex2 (1 - exp(-x) rounds to
//               1.0f for every pair), one-float coordinates relative to the
//               group centre;
//   P2P_FULL:   the other sources beyond the series radius sqrt(r2_series):
//               no small-x check (every pair has r2 above r2_series);
//   P2P_SERIES: the sources within it: the pair code with the check.
// Full and series pairs give bitwise the value of the checked code.  The group's
// sources stream through three warp buffers, one per mode (each in stream
// order), and each buffer runs 32 sources at a time as it fills (the rest
// when the group's stream ends).
constexpr int P2P_FAR = 0, P2P_FULL = 1, P2P_SERIES = 2;

template <int MODE>
__device__ __forceinline__ void scalar_pair(const ulonglong2 &h, const ulonglong2 &l,
                                            unsigned long long g2, const float4 &t,
                                            const pfd::GaussParams &gp, float &px, float &py) {
    float sxh, syh, sxl, syl, g, dummy;
    pfd::unpack2(h.x, sxh, dummy);
    pfd::unpack2(h.y, syh, dummy);
    pfd::unpack2(l.x, sxl, dummy);
    pfd::unpack2(l.y, syl, dummy);
    pfd::unpack2(g2, g, dummy);
    const float dx = (t.x - sxh) + (t.z - sxl);
    const float dy = (t.y - syh) + (t.w - syl);
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, 1e-12f));
    const float sc = MODE == P2P_FAR ? g * pfd::rcp_approx(r2)
                                     : pfd::gauss_s<MODE == P2P_SERIES>(r2, g, gp);
    px = fmaf(-dy, sc, px);
    py = fmaf(dx, sc, py);
}

// One pair of the given mode for the lane's targets (NT per lane).
template <int NT, int MODE>
__device__ __forceinline__ void p2p_pair(const ulonglong2 &h, const ulonglong2 &l,
                                         unsigned long long g2, pfd::f32x2 txh, pfd::f32x2 tyh,
                                         pfd::f32x2 txl, pfd::f32x2 tyl, const float4 &ta,
                                         const float4 &tc, const pfd::GaussParams &gp,
                                         const pfd::GaussParams2 &gp2, pfd::f32x2 &nx,
                                         pfd::f32x2 &ny, float &pxa, float &pya, float &pxc,
                                         float &pyc) {
    if (NT >= 2) {
        if (MODE == P2P_FAR)
            pfd::pair2_far(h, l, g2, txh, tyh, txl, tyl, gp2, nx, ny);
        else
            pfd::pair2<MODE == P2P_SERIES>(h, l, g2, txh, tyh, txl, tyl, gp2, nx, ny);
    } else {
        scalar_pair<MODE>(h, l, g2, ta, gp, pxa, pya);
    }
    if (NT == 3) scalar_pair<MODE>(h, l, g2, tc, gp, pxc, pyc);
}

// Shared-memory loads by 32-bit shared address (the chunk functions below
// are separate calls, which see only generic pointers otherwise).
__device__ __forceinline__ ulonglong2 lds_u64x2(uint32_t a) {
    ulonglong2 v;
    asm("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ unsigned long long lds_u64(uint32_t a) {
    unsigned long long v;
    asm("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(a));
    return v;
}

struct P2PSums {
    float s[6];  // NT >= 2: -nx_a, ny_a, -nx_b, ny_b; NT = 1: px_a, py_a; NT = 3: px_c, py_c
};

// Sources [0, cnt) of a buffer (cnt <= 32) against the lane's targets; the
// partial sums are returned for one compensated fold by the caller.  Each
// (NT, MODE) is its own function, not inlined: nine inlined copies of the
// unrolled loop in one kernel measured about 20% more instructions (register
// copies between the copies' allocations) and instruction-cache stalls.
// (A per-source choice of the checked code inside a chunk, by a warp-uniform
// branch, measured slower too: the branch breaks the overlap of consecutive
// pairs.)
//
// P2P_FAR chunks hold coordinates relative to the group centre (cx, cy), one
// float each: {x - cx, x - cx, y - cy, y - cy} in the hi slot (pair2_far_local).
__device__ __forceinline__ void far_local_scalar(const ulonglong2 &loc, unsigned long long g2,
                                                 float tx, float ty, float &px, float &py) {
    float lx, ly, g, dummy;
    pfd::unpack2(loc.x, lx, dummy);
    pfd::unpack2(loc.y, ly, dummy);
    pfd::unpack2(g2, g, dummy);
    const float dx = tx - lx, dy = ty - ly;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, 1e-12f));
    const float sc = g * pfd::rcp_approx(r2);
    px = fmaf(-dy, sc, px);
    py = fmaf(dx, sc, py);
}

template <int NT, int MODE>
__device__ __noinline__ P2PSums p2p_chunk_sums(uint32_t a_hi, uint32_t a_lo, uint32_t a_g, int cnt,
                                               float4 ta, float4 tb, float4 tc, float cx,
                                               float cy, pfd::GaussParams gp) {
    const pfd::GaussParams2 gp2 = pfd::make_params2(gp);
    pfd::f32x2 nx = 0ull, ny = 0ull;  // +0.0f in both halves
    float pxa = 0.f, pya = 0.f, pxc = 0.f, pyc = 0.f;
    if constexpr (MODE == P2P_FAR) {
        const float axc = (ta.x - cx) + ta.z, ayc = (ta.y - cy) + ta.w;
        const pfd::f32x2 txc = pfd::pack2(axc, (tb.x - cx) + tb.z);
        const pfd::f32x2 tyc = pfd::pack2(ayc, (tb.y - cy) + tb.w);
        auto one = [&](int k) {
            const ulonglong2 loc = lds_u64x2(a_hi + 16 * k);
            const unsigned long long g2 = lds_u64(a_g + 8 * k);
            if (NT >= 2)
                pfd::pair2_far_local(loc, g2, txc, tyc, gp2, nx, ny);
            else
                far_local_scalar(loc, g2, axc, ayc, pxa, pya);
        };
        if (cnt == 32) {
#pragma unroll(P2P_UNROLL)
            for (int k = 0; k < 32; ++k) one(k);
        } else {
#pragma unroll 1
            for (int k = 0; k < cnt; ++k) one(k);
        }
    } else {
        const pfd::f32x2 txh = pfd::pack2(ta.x, tb.x), tyh = pfd::pack2(ta.y, tb.y);
        const pfd::f32x2 txl = pfd::pack2(ta.z, tb.z), tyl = pfd::pack2(ta.w, tb.w);
        if (cnt == 32) {  // full chunk (the common case)
#pragma unroll(P2P_UNROLL)
            for (int k = 0; k < 32; ++k)
                p2p_pair<NT, MODE>(lds_u64x2(a_hi + 16 * k), lds_u64x2(a_lo + 16 * k),
                                   lds_u64(a_g + 8 * k), txh, tyh, txl, tyl, ta, tc, gp, gp2, nx,
                                   ny, pxa, pya, pxc, pyc);
        } else {  // the rest of a buffer at the end of a group: kept small in code
#pragma unroll 1
            for (int k = 0; k < cnt; ++k)
                p2p_pair<NT, MODE>(lds_u64x2(a_hi + 16 * k), lds_u64x2(a_lo + 16 * k),
                                   lds_u64(a_g + 8 * k), txh, tyh, txl, tyl, ta, tc, gp, gp2, nx,
                                   ny, pxa, pya, pxc, pyc);
        }
    }
    P2PSums r;
    if (NT >= 2) {
        float nxa, nxb, nya, nyb;
        pfd::unpack2(nx, nxa, nxb);
        pfd::unpack2(ny, nya, nyb);
        r.s[0] = -nxa;
        r.s[1] = nya;
        r.s[2] = -nxb;
        r.s[3] = nyb;
    } else {
        r.s[0] = pxa;
        r.s[1] = pya;
        r.s[2] = r.s[3] = 0.f;
    }
    r.s[4] = pxc;
    r.s[5] = pyc;
    return r;
}

template <int NT, int MODE>
__device__ __forceinline__ void p2p_chunk(const ulonglong2 *shi, const ulonglong2 *slo,
                                          const unsigned long long *sg2, int cnt,
                                          const float4 &ta, const float4 &tb, const float4 &tc,
                                          float cx, float cy, const pfd::GaussParams &gp,
                                          float (&acc)[16]) {
    const P2PSums r = p2p_chunk_sums<NT, MODE>(
        (uint32_t)__cvta_generic_to_shared(shi), (uint32_t)__cvta_generic_to_shared(slo),
        (uint32_t)__cvta_generic_to_shared(sg2), cnt, ta, tb, tc, cx, cy, gp);
    pfd::comp_add(acc[0], acc[1], r.s[0]);
    pfd::comp_add(acc[2], acc[3], r.s[1]);
    if (NT >= 2) {
        pfd::comp_add(acc[4], acc[5], r.s[2]);
        pfd::comp_add(acc[6], acc[7], r.s[3]);
    }
    if (NT == 3) {
        pfd::comp_add(acc[8], acc[9], r.s[4]);
        pfd::comp_add(acc[10], acc[11], r.s[5]);
    }
}

// The third target slot of a group of 65..96 targets: the rem = size - 64
// remainder targets are paired (c, d) into rp = ceil(rem / 2) packed pairs
// spread over the warp, m = 32 / rp lanes per pair, lane (j + rp q) taking
// sources q, q + m, q + 2m, ... of the chunk for pair j with the packed pair
// code of the main slots; the m partial sums are combined at the end of the
// group.  Lanes with no share get q >= 32.  Returns -nx_c, ny_c, -nx_d, ny_d.
template <int MODE>
__device__ __noinline__ float4 p2p_split_sums(uint32_t a_hi, uint32_t a_lo, uint32_t a_g, int cnt,
                                              int q, int m, float4 tc, float4 td, float cx,
                                              float cy, pfd::GaussParams gp) {
    const pfd::GaussParams2 gp2 = pfd::make_params2(gp);
    pfd::f32x2 nx = 0ull, ny = 0ull;
    if constexpr (MODE == P2P_FAR) {
        const pfd::f32x2 txc = pfd::pack2((tc.x - cx) + tc.z, (td.x - cx) + td.z);
        const pfd::f32x2 tyc = pfd::pack2((tc.y - cy) + tc.w, (td.y - cy) + td.w);
#pragma unroll 2
        for (int k = q; k < cnt; k += m)
            pfd::pair2_far_local(lds_u64x2(a_hi + 16 * k), lds_u64(a_g + 8 * k), txc, tyc, gp2, nx,
                                 ny);
    } else {
        const pfd::f32x2 txh = pfd::pack2(tc.x, td.x), tyh = pfd::pack2(tc.y, td.y);
        const pfd::f32x2 txl = pfd::pack2(tc.z, td.z), tyl = pfd::pack2(tc.w, td.w);
#pragma unroll 2
        for (int k = q; k < cnt; k += m)
            pfd::pair2<MODE == P2P_SERIES>(lds_u64x2(a_hi + 16 * k), lds_u64x2(a_lo + 16 * k),
                                            lds_u64(a_g + 8 * k), txh, tyh, txl, tyl, gp2, nx, ny);
    }
    float nxc, nxd, nyc, nyd;
    pfd::unpack2(nx, nxc, nxd);
    pfd::unpack2(ny, nyc, nyd);
    return make_float4(-nxc, nyc, -nxd, nyd);
}

// p2p_chunk for the group's targets-per-lane count nt (warp-uniform).
// nt = 3: targets a, b packed plus the lane's share (qs of msp) of a
// remainder target pair (c, d).
template <int MODE>
__device__ __forceinline__ void p2p_run_chunk(int nt, const ulonglong2 *shi, const ulonglong2 *slo,
                                              const unsigned long long *sg2, int cnt,
                                              const float4 &ta, const float4 &tb,
                                              const float4 &tc, const float4 &td, int qs,
                                              int msp, float cx, float cy,
                                              const pfd::GaussParams &gp, float (&acc)[16]) {
    if (nt == 1) {
        p2p_chunk<1, MODE>(shi, slo, sg2, cnt, ta, tb, tc, cx, cy, gp, acc);
        return;
    }
    p2p_chunk<2, MODE>(shi, slo, sg2, cnt, ta, tb, tc, cx, cy, gp, acc);
    if (nt == 3) {
        const float4 r = p2p_split_sums<MODE>(
            (uint32_t)__cvta_generic_to_shared(shi), (uint32_t)__cvta_generic_to_shared(slo),
            (uint32_t)__cvta_generic_to_shared(sg2), cnt, qs, msp, tc, td, cx, cy, gp);
        pfd::comp_add(acc[8], acc[9], r.x);
        pfd::comp_add(acc[10], acc[11], r.y);
        pfd::comp_add(acc[12], acc[13], r.z);
        pfd::comp_add(acc[14], acc[15], r.w);
    }
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

constexpr int P2P_OWN_GROUPS = 4;  // target groups a block's own CTA computes at most


// Target group gi of block b (groups of at most 96 targets, balanced: sizes
// differ by at most one; every group streams all the block's sources, so a
// small last group would cost nearly as much as a full one) against the
// block's whole source stream; writes the group's near-field velocities.
__device__ __forceinline__ void p2p_group_body(
    int64_t b, int t0, int tn, int ngrp, int gi, const int32_t *__restrict__ sstart,
    const int32_t *__restrict__ scnt, const float4 *__restrict__ shl,
    const float *__restrict__ sg32, const float4 *__restrict__ thl,
    const int32_t *__restrict__ run_off, const int2 *__restrict__ runs, pfd::GaussParams gp,
    double2 *__restrict__ nearv, ulonglong2 (*s_hi)[P2P_BUF], ulonglong2 (*s_lo)[P2P_BUF],
    unsigned long long (*s_g2)[P2P_BUF], int *s_rs, int *s_rp, unsigned long long &npairs,
    unsigned long long &nfar, int64_t ns_all, int64_t nt_all) {
    const int lane = threadIdx.x;
    const unsigned lt = (1u << lane) - 1u;
    const float rser = sqrtf(gp.r2_series);
    const int r0 = run_off[b], r1 = run_off[b + 1];
    const int tg = (int)((int64_t)gi * tn / ngrp);
    const int gsz = (int)((int64_t)(gi + 1) * tn / ngrp) - tg;
    const int nt = (gsz <= 32) ? 1 : (gsz <= 64) ? 2 : 3;  // warp-uniform
    // nt = 3: remainder targets tg + 64 + j, j < rem, in rp packed pairs
    // (tg + 64 + 2 p, + 1), each pair on msp lanes
    const int rem = nt == 3 ? gsz - 64 : 32;
    const int rp = (rem + 1) / 2;
    const int msp = 32 / rp;
    const bool cval = nt == 3 && lane < rp * msp;
    const int qs = cval ? lane / rp : 32;
    const int ia = tg + lane, ib = tg + 32 + lane, ic = tg + 64 + 2 * (lane % rp), id = ic + 1;
    const bool dval = cval && id < tg + gsz;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!PF_IDX_OK((int64_t)t0 + tg + gsz - 1, nt_all, 204)) return;  // the group's last target
    const float4 ta = (lane < gsz) ? thl[t0 + ia] : z4;
    const float4 tb = (lane + 32 < gsz) ? thl[t0 + ib] : z4;
    const float4 tc = cval ? thl[t0 + ic] : z4;
    const float4 td = dval ? thl[t0 + id] : tc;  // an odd remainder's last pair repeats c
    // box of the group's targets (hi parts), for the series-free test
    float bx0 = INFINITY, bx1 = -INFINITY, by0 = INFINITY, by1 = -INFINITY;
    if (lane < gsz) { bx0 = bx1 = ta.x; by0 = by1 = ta.y; }
    if (lane + 32 < gsz) { bx0 = fminf(bx0, tb.x); bx1 = fmaxf(bx1, tb.x); by0 = fminf(by0, tb.y); by1 = fmaxf(by1, tb.y); }
    if (cval) { bx0 = fminf(bx0, fminf(tc.x, td.x)); bx1 = fmaxf(bx1, fmaxf(tc.x, td.x)); by0 = fminf(by0, fminf(tc.y, td.y)); by1 = fmaxf(by1, fmaxf(tc.y, td.y)); }
    bx0 = warp_min(bx0);
    bx1 = warp_max(bx1);
    by0 = warp_min(by0);
    by1 = warp_max(by1);
    // a source at box distance d has r2 >= (d - e)^2 for every target, e
    // covering the hi-part rounding of both points (2^-23 relative each)
    const float mag = fmaxf(fmaxf(fabsf(bx0), fabsf(bx1)), fmaxf(fabsf(by0), fabsf(by1)));
    const float reach = rser * 1.001f + (mag + rser) * 4.8e-7f + 1e-30f;
    const float reach2 = reach * reach;
    const float rfar = sqrtf(gp.r2_far);
    const float reachf = rfar * 1.001f + (mag + rfar) * 4.8e-7f + 1e-30f;
    const float reachf2 = reachf * reachf;
    // centre for the far sources' relative coordinates (any float near the group)
    const float cx = 0.5f * (bx0 + bx1), cy = 0.5f * (by0 + by1);
    float acc[16] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f,
                     0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    // the three buffers are rings of P2P_BUF = 64 entries: entries waiting
    // c0, c1, c2 from heads h0, h1, h2; a chunk is always the 32 entries at
    // the head (0 or 32), so it never wraps, and taking it flips the head
    int c0 = 0, c1 = 0, c2 = 0;
    int h0 = 0, h1 = 0, h2 = 0;
    for (int rc = r0; rc < r1; rc += P2P_RUNS_SM) {
        const int nrc = min(P2P_RUNS_SM, r1 - rc);
        int pre = 0;
        for (int k0 = 0; k0 < nrc; k0 += 32) {
            const int k = k0 + lane;
            int st = 0, len = 0;
            if (k < nrc) {
                const int2 rr = runs[rc + k];
                st = sstart[rr.x];
                len = sstart[rr.y] + scnt[rr.y] - st;
            }
            int inc = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            if (k < nrc) {
                s_rs[k] = st;
                s_rp[k] = pre + inc - len;
            }
            pre += __shfl_sync(0xffffffffu, inc, 31);
        }
        if (lane == 0) s_rp[nrc] = pre;
        __syncwarp();
        const int S = pre;
        npairs += (unsigned long long)S * (unsigned long long)gsz;
        // each lane's stream position only moves forward (by 32 per
        // round), so the run holding it is found by advancing an index:
        // the largest r with prefix[r] <= p (empty runs are stepped over).
        // The loads of round s0 + 32 are issued before round s0's chunks
        // run, so their latency overlaps the pair work.
        int rr = 0;
        float4 spv = z4;
        float gg = 0.f;
        auto fetch = [&](int p, float4 &v, float &w) {
            if (p < S) {
                while (rr + 1 < nrc && s_rp[rr + 1] <= p) ++rr;
                const int src = s_rs[rr] + (p - s_rp[rr]);
                if (PF_IDX_OK(src, ns_all, 203)) {
                    v = shl[src];
                    w = sg32[src];
                }
            }
        };
        fetch(lane, spv, gg);
        for (int s0 = 0; s0 < S; s0 += 32) {
            const int p = s0 + lane;
            int cls = -1;  // 0 far, 1 full, 2 series; -1 past the stream
            if (p < S) {
                const float ex = fmaxf(fmaxf(bx0 - spv.x, spv.x - bx1), 0.f);
                const float ey = fmaxf(fmaxf(by0 - spv.y, spv.y - by1), 0.f);
                const float d2 = ex * ex + ey * ey;
                cls = d2 > reachf2 ? 0 : d2 > reach2 ? 1 : 2;
            }
            // append each source to the buffer of its mode, in stream order
            const unsigned m0 = __ballot_sync(0xffffffffu, cls == 0);
            const unsigned m1 = __ballot_sync(0xffffffffu, cls == 1);
            const unsigned m2 = __ballot_sync(0xffffffffu, cls == 2);
            if (cls >= 0) {
                const unsigned mm = cls == 0 ? m0 : cls == 1 ? m1 : m2;
                const int k =
                    ((cls == 0 ? h0 + c0 : cls == 1 ? h1 + c1 : h2 + c2) + __popc(mm & lt)) &
                    (P2P_BUF - 1);
                if (cls == 0) {  // far: coordinates relative to the group centre
                    const float lx = (spv.x - cx) + spv.z, ly = (spv.y - cy) + spv.w;
                    s_hi[0][k] = make_ulonglong2(pfd::pack2(lx, lx), pfd::pack2(ly, ly));
                } else {
                    s_hi[cls][k] = make_ulonglong2(pfd::pack2(spv.x, spv.x),
                                                   pfd::pack2(spv.y, spv.y));
                    s_lo[cls][k] = make_ulonglong2(pfd::pack2(spv.z, spv.z),
                                                   pfd::pack2(spv.w, spv.w));
                }
                s_g2[cls][k] = pfd::pack2(gg, gg);
            }
            c0 += __popc(m0);
            c1 += __popc(m1);
            c2 += __popc(m2);
            spv = z4;
            gg = 0.f;
            fetch(p + 32, spv, gg);
            __syncwarp();
            bool ran = false;  // warp-uniform
            if (c0 >= 32) {
                p2p_run_chunk<P2P_FAR>(nt, s_hi[0] + h0, s_lo[0] + h0, s_g2[0] + h0, 32, ta, tb,
                                       tc, td, qs, msp, cx, cy, gp, acc);
                nfar += 32ull * (unsigned long long)gsz;
                c0 -= 32;
                h0 ^= 32;
                ran = true;
            }
            if (c1 >= 32) {
                p2p_run_chunk<P2P_FULL>(nt, s_hi[1] + h1, s_lo[1] + h1, s_g2[1] + h1, 32, ta,
                                        tb, tc, td, qs, msp, cx, cy, gp, acc);
                c1 -= 32;
                h1 ^= 32;
                ran = true;
            }
            if (c2 >= 32) {
                p2p_run_chunk<P2P_SERIES>(nt, s_hi[2] + h2, s_lo[2] + h2, s_g2[2] + h2, 32, ta,
                                          tb, tc, td, qs, msp, cx, cy, gp, acc);
                c2 -= 32;
                h2 ^= 32;
                ran = true;
            }
            if (ran) __syncwarp();  // the chunks are read before the next round refills them
        }
    }
    // what is left in the buffers (fewer than 32 each)
    // (fewer than 32 from a head of 0 or 32: no wrap)
    if (c0)
        p2p_run_chunk<P2P_FAR>(nt, s_hi[0] + h0, s_lo[0] + h0, s_g2[0] + h0, c0, ta, tb, tc,
                               td, qs, msp, cx, cy, gp, acc);
    nfar += (unsigned long long)c0 * (unsigned long long)gsz;
    if (c1)
        p2p_run_chunk<P2P_FULL>(nt, s_hi[1] + h1, s_lo[1] + h1, s_g2[1] + h1, c1, ta, tb, tc,
                                td, qs, msp, cx, cy, gp, acc);
    if (c2)
        p2p_run_chunk<P2P_SERIES>(nt, s_hi[2] + h2, s_lo[2] + h2, s_g2[2] + h2, c2, ta, tb,
                                  tc, td, qs, msp, cx, cy, gp, acc);
    __syncwarp();
    if (lane < gsz)
        nearv[t0 + ia] = make_double2(INV_2PI * ((double)acc[0] + (double)acc[1]),
                                      INV_2PI * ((double)acc[2] + (double)acc[3]));
    if (lane + 32 < gsz)
        nearv[t0 + ib] = make_double2(INV_2PI * ((double)acc[4] + (double)acc[5]),
                                      INV_2PI * ((double)acc[6] + (double)acc[7]));
    if (nt == 3) {  // combine the msp shares of each remainder pair, in lane order
        float h[4] = {acc[8], acc[10], acc[12], acc[14]};
        float l[4] = {acc[9], acc[11], acc[13], acc[15]};
        for (int q = 1; q < msp; ++q) {
            const int sl = lane % rp + rp * q;  // < rp * msp <= 32
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const float a = __shfl_sync(0xffffffffu, acc[8 + 2 * v], sl);
                const float b = __shfl_sync(0xffffffffu, acc[9 + 2 * v], sl);
                pfd::comp_add(h[v], l[v], a);
                l[v] += b;
            }
        }
        if (lane < rp) {
            nearv[t0 + ic] = make_double2(INV_2PI * ((double)h[0] + (double)l[0]),
                                          INV_2PI * ((double)h[1] + (double)l[1]));
            if (dval)
                nearv[t0 + id] = make_double2(INV_2PI * ((double)h[2] + (double)l[2]),
                                              INV_2PI * ((double)h[3] + (double)l[3]));
        }
    }
}

// Shared memory of one P2P CTA (one warp).
struct P2PSmem {
    // source buffers, one per mode: [P2P_FAR], [P2P_FULL], [P2P_SERIES]
    ulonglong2 hi[3][P2P_BUF];  // {x_hi, x_hi}, {y_hi, y_hi}
    ulonglong2 lo[3][P2P_BUF];  // {x_lo, x_lo}, {y_lo, y_lo}
    unsigned long long g2[3][P2P_BUF];  // {g, g}
    int rs[P2P_RUNS_SM];      // particle start of run
    int rp[P2P_RUNS_SM + 1];  // stream prefix of run
};

// Targets of P2P block b: first sorted target t0, count returned.
__device__ __forceinline__ int p2p_targets(const P2PDesc &d, int64_t b, int &t0) {
    const uint32_t leaf0 = (uint32_t)b << (2 * d.kb), nl = 1u << (2 * d.kb);
    t0 = d.tstart[leaf0];
    return d.tstart[leaf0 + nl - 1] + d.tcnt[leaf0 + nl - 1] - t0;
}

__device__ __forceinline__ void p2p_group(const P2PDesc &d, int64_t b, int t0, int tn, int ngrp,
                                          int gi, P2PSmem &sm, unsigned long long &npairs,
                                          unsigned long long &nfar) {
    p2p_group_body(b, t0, tn, ngrp, gi, d.sstart, d.scnt, d.shl, d.sg32, d.thl, d.run_off, d.runs,
                   d.gp, d.nearv, sm.hi, sm.lo, sm.g2, sm.rs, sm.rp, npairs, nfar, d.work.ns,
                   d.work.nt);
}

// The CTA of P2P block `local` (launch order): its target groups, unless
// there are more than P2P_OWN_GROUPS of them: such a block (a dense cluster)
// is listed as heavy for the second launch.
__device__ __forceinline__ void p2p_own_block(const P2PDesc &d, int64_t local, P2PSmem &sm,
                                              unsigned long long &npairs,
                                              unsigned long long &nfar) {
    const int64_t b = d.order[local];
    int t0;
    const int tn = p2p_targets(d, b, t0);
    if (tn == 0) return;
    const int ngrp = (tn + 95) / 96;
    if (ngrp > P2P_OWN_GROUPS) {  // left to the second launch
        if (threadIdx.x == 0) d.work.heavy[atomicAdd(d.work.heavy_n, 1u)] = (int32_t)b;
    } else {
        for (int gi = 0; gi < ngrp; ++gi) p2p_group(d, b, t0, tn, ngrp, gi, sm, npairs, nfar);
    }
}

// The groups of one heavy block, shared out through its counter (counters
// only, no waits; each group is computed by exactly one CTA, so results do
// not depend on the schedule).
__device__ __forceinline__ void p2p_heavy_block(const P2PDesc &d, int64_t b, P2PSmem &sm,
                                                unsigned long long &npairs,
                                                unsigned long long &nfar) {
    int t0;
    const int tn = p2p_targets(d, b, t0);
    const int ngrp = (tn + 95) / 96;
    for (;;) {
        unsigned gi = 0;
        if (threadIdx.x == 0) gi = atomicAdd((unsigned *)&d.work.grp_next[b], 1u);
        gi = __shfl_sync(0xffffffffu, gi, 0);
        if ((int)gi >= ngrp) break;
        p2p_group(d, b, t0, tn, ngrp, (int)gi, sm, npairs, nfar);
    }
}

__device__ __forceinline__ void p2p_heavy_blocks(const P2PDesc &d, P2PSmem &sm,
                                                 unsigned long long &npairs,
                                                 unsigned long long &nfar) {
    const unsigned nh = *d.work.heavy_n;  // complete: written by the first launch
    for (unsigned k = 0; k < nh; ++k) p2p_heavy_block(d, d.work.heavy[k], sm, npairs, nfar);
}

__device__ __forceinline__ void p2p_count(const P2PDesc &d, unsigned long long npairs,
                                          unsigned long long nfar) {
    if (threadIdx.x == 0 && (npairs | nfar)) {
        atomicAdd(d.pairs, npairs);
        atomicAdd(d.pairs + 2, nfar);
    }
}

// Two launches of one kernel.  HEAVY = false: one CTA per P2P block (in
// launch order) computes the block's target groups (or lists the block as
// heavy).  HEAVY = true: persistent CTAs share out the groups of the heavy
// blocks.  Without dense clusters the second launch finds nothing to do.
template <bool HEAVY>
__global__ void __launch_bounds__(32, P2P_MIN_CTAS) k_p2p(const P2PDesc d) {
    __shared__ P2PSmem sm;
    unsigned long long npairs = 0, nfar = 0;
    if (!HEAVY) {
        if ((int64_t)blockIdx.x >= d.nblk) return;
        p2p_own_block(d, blockIdx.x, sm, npairs, nfar);
    } else {
        p2p_heavy_blocks(d, sm, npairs, nfar);
    }
    p2p_count(d, npairs, nfar);
}

// SMs of the current device (cached per device; host threads may race to
// fill an entry, all with the same value).
static int p2p_sm_count() {
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cached[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// L2P + near + scatter to input order: one thread per sorted target
template <int NP>
__global__ void __launch_bounds__(256)
k_l2p(int64_t nt, int L, double x0, double y0, double wl, const double *__restrict__ tx,
      const double *__restrict__ ty, const uint32_t *__restrict__ tkey_sorted,
      const double2 *__restrict__ Lc, const double2 *__restrict__ nearv,
      const int32_t *__restrict__ perm, double *__restrict__ vx, double *__restrict__ vy) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= nt) return;
    const uint32_t m = tkey_sorted[i];
    const uint32_t ix = compact1by1(m), iy = compact1by1(m >> 1);
    const double iw = 1.0 / wl;
    const double2 z = make_double2((tx[i] - (x0 + ((double)ix + 0.5) * wl)) * iw,
                                   (ty[i] - (y0 + ((double)iy + 0.5) * wl)) * iw);
    const double2 *lam = Lc + (level_off(L) + m) * NP;
    double2 w = lam[NP - 1];
#pragma unroll
    for (int n = NP - 2; n >= 0; --n) w = cfma(w, z, lam[n]);
    const double2 nv = nearv[i];
    const int32_t o = perm[i];
    if (!PF_IDX_OK(o, nt, 205)) return;
    vx[o] = nv.x + INV_2PI * iw * w.y;
    vy[o] = nv.y + INV_2PI * iw * w.x;
}


// ---------------------------------------------------------------------------
// Host: plan cache (tables + operators on the device)
struct FmmCache {
    int L = -1, kb = -1, np = -1;
    double ratio = -1.0;       // cutoff / root width the tables were built with
    std::vector<int64_t> sep;  // separation key of those tables (fmm_plan.cuh)
    int maxpos = 0, nq = 0, nqp = 0;
    int4 *d_far = nullptr;
    int32_t *d_far_ptr = nullptr;
    int2 *d_q = nullptr;
    int32_t *d_run_off = nullptr;  // [nblk + 1]
    int2 *d_runs = nullptr;        // (first, last) leaf of each run
    int32_t *d_blk_order = nullptr;  // P2P block launch order (heaviest first)
    int64_t nruns = 0;
    size_t dev_bytes = 0;          // device memory held by this plan
    size_t bytes() const { return dev_bytes; }
    double2 *d_pw = nullptr;
    double *d_m2m = nullptr, *d_l2l = nullptr;  // tensor-core fragment tables
    double *d_bin = nullptr;
    void release() {
        cudaFree(d_far);
        cudaFree(d_far_ptr);
        cudaFree(d_q);
        cudaFree(d_pw);
        cudaFree(d_m2m);
        cudaFree(d_l2l);
        cudaFree(d_bin);
        cudaFree(d_run_off);
        cudaFree(d_runs);
        cudaFree(d_blk_order);
        d_blk_order = nullptr;
        d_run_off = nullptr;
        d_runs = nullptr;
        d_far = nullptr;
        d_far_ptr = nullptr;
        d_q = nullptr;
        d_pw = nullptr;
        d_m2m = d_l2l = nullptr;
        d_bin = nullptr;
        L = -1;
    }
};

struct cplx {
    double re, im;
};
static cplx cm(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

static double binom_d(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1.0;  // exact while the value stays below 2^53
    for (int i = 1; i <= k; ++i) r = r * (double)(n - k + i) / (double)i;
    return r;
}

template <typename T>
static pf_status upload(T **dst, const std::vector<T> &v, size_t &tally) {
    if (v.empty()) {
        *dst = nullptr;
        return PF_OK;
    }
    tally += sizeof(T) * v.size();
    PF_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(dst), sizeof(T) * v.size()));
    PF_CUDA_TRY(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return PF_OK;
}

static std::atomic<uint64_t> g_plan_builds{0};  // plans built in this process

static pf_status build_cache(FmmCache &c, int L, int kb, int np, double w0, double cutoff) {
    c.release();
    size_t tally = 0;
    pf::fmm::Tables t;
    pf::fmm::build_tables(L, kb, w0, cutoff, THETA, t);
    const int B = 1 << kb, Bp = B > 2 ? B : 2;
    c.maxpos = std::max(4, Bp * Bp);
    // far lists with offset ids
    std::vector<int4> far;
    std::vector<int32_t> ptr((L + 1) * c.maxpos + 1, 0);
    std::vector<pf::fmm::Off> ops;
    auto op_id = [&](const pf::fmm::Off &o) {
        for (size_t k = 0; k < ops.size(); ++k)
            if (ops[k] == o) return (int)k;
        ops.push_back(o);
        return (int)ops.size() - 1;
    };
    for (int l = 0; l <= L; ++l) {
        for (int p = 0; p < c.maxpos; ++p) {
            ptr[l * c.maxpos + p] = (int32_t)far.size();
            if (l >= 2 && p < (int)t.far[l].size())
                for (const auto &o : t.far[l][p]) {
                    // .w: the offset in Morton-dilated form (two's complement per
                    // coordinate, 16 bits each), for morton_add in k_m2l
                    const uint32_t d = morton2((uint32_t)o.i & 0xffffu, (uint32_t)o.j & 0xffffu);
                    far.push_back(make_int4(o.i, o.j, op_id(o), (int)d));
                }
        }
    }
    ptr[(L + 1) * c.maxpos] = (int32_t)far.size();  // [l*maxpos + pos] .. next slot
    // powers rho^m, m = 0..np, rho = 1/(i + i j)
    std::vector<double2> pw(ops.size() * (np + 1));
    for (size_t k = 0; k < ops.size(); ++k) {
        const double i = ops[k].i, j = ops[k].j, d = i * i + j * j;
        const cplx rho = {i / d, -j / d};
        cplx pm = {1.0, 0.0};
        for (int m = 0; m <= np; ++m) {
            pw[k * (np + 1) + m] = make_double2(pm.re, pm.im);
            pm = cm(pm, rho);
        }
    }
    // M2M / L2L operators, stored transposed for coalesced lane access
    std::vector<double2> m2m(4 * np * np), l2l(4 * np * np);
    for (int cc = 0; cc < 4; ++cc) {
        const cplx tau = {(cc & 1) ? 0.25 : -0.25, (cc & 2) ? 0.25 : -0.25};
        std::vector<cplx> tp(np);
        tp[0] = {1.0, 0.0};
        for (int k = 1; k < np; ++k) tp[k] = cm(tp[k - 1], tau);
        for (int k = 0; k < np; ++k)
            for (int m = 0; m < np; ++m) {
                // M2M: out k, in m (m <= k): C(k,m) tau^(k-m) 2^-m   -> opT[c][m][k]
                cplx a = {0.0, 0.0};
                if (m <= k) {
                    const double s = binom_d(k, m) * std::ldexp(1.0, -m);
                    a = {tp[k - m].re * s, tp[k - m].im * s};
                }
                m2m[(size_t)cc * np * np + (size_t)m * np + k] = make_double2(a.re, a.im);
                // L2L: out n = k, in m (m >= n): 1/2 C(m,n) tau^(m-n) 2^-n -> opT[c][m][n]
                cplx b = {0.0, 0.0};
                if (m >= k) {
                    const double s = 0.5 * binom_d(m, k) * std::ldexp(1.0, -k);
                    b = {tp[m - k].re * s, tp[m - k].im * s};
                }
                l2l[(size_t)cc * np * np + (size_t)m * np + k] = make_double2(b.re, b.im);
            }
    }
    // the same operators as A-operand fragment tables of the tensor-core
    // kernels: [c][part][mt][ks][lane] = part of T_c[8 mt + lane/4][4 ks + lane%4]
    // with T_c[k][m] = m2m[c][m][k] (M2M) and T_c[n][m] = l2l[c][m][n] (L2L)
    const int MTh = (np + 7) / 8, KSh = (np + 3) / 4;
    std::vector<double> m2mf(4 * 2 * MTh * KSh * 32), l2lf(m2mf.size());
    for (int cc = 0; cc < 4; ++cc)
        for (int part = 0; part < 2; ++part)
            for (int mt = 0; mt < MTh; ++mt)
                for (int ks = 0; ks < KSh; ++ks)
                    for (int ln = 0; ln < 32; ++ln) {
                        const int row = 8 * mt + ln / 4, col = 4 * ks + ln % 4;
                        const size_t o = ((((size_t)cc * 2 + part) * MTh + mt) * KSh + ks) * 32 + ln;
                        double vm = 0.0, vl = 0.0;
                        if (row < np && col < np) {
                            const double2 a = m2m[(size_t)cc * np * np + (size_t)col * np + row];
                            const double2 b = l2l[(size_t)cc * np * np + (size_t)col * np + row];
                            vm = part ? a.y : a.x;
                            vl = part ? b.y : b.x;
                        }
                        m2mf[o] = vm;
                        l2lf[o] = vl;
                    }
    std::vector<double> bin(np * np);
    for (int k = 0; k < np; ++k)
        for (int n = 0; n < np; ++n) bin[k * np + n] = binom_d(n + k, k);
    std::vector<int2> q;
    for (const auto &o : t.p2p) q.push_back(make_int2(o.i, o.j));
    c.nq = (int)q.size();
    c.nqp = 1;
    while (c.nqp < c.nq) c.nqp <<= 1;
    PF_TRY(upload(&c.d_far, far, tally));
    PF_TRY(upload(&c.d_far_ptr, ptr, tally));
    PF_TRY(upload(&c.d_q, q, tally));
    PF_TRY(upload(&c.d_pw, pw, tally));
    PF_TRY(upload(&c.d_m2m, m2mf, tally));
    PF_TRY(upload(&c.d_l2l, l2lf, tally));
    PF_TRY(upload(&c.d_bin, bin, tally));
    if (c.nqp <= P2P_QMAX) {
        // P2P run lists of every block (geometry only, reused by every call)
        const int64_t nblk = (int64_t)1 << (2 * (L - kb));
        PF_CUDA_TRY(cudaMalloc(&c.d_run_off, sizeof(int32_t) * (nblk + 1)));
        k_p2p_runs<<<(unsigned)nblk, P2P_SETUP_THREADS>>>(L, kb, c.d_q, c.nq, c.nqp, c.d_run_off,
                                                          nullptr);
        PF_TRY(pf::launch_status("k_p2p_runs"));
        std::vector<int32_t> cnt(nblk + 1, 0);
        PF_CUDA_TRY(cudaMemcpy(cnt.data(), c.d_run_off, sizeof(int32_t) * nblk,
                               cudaMemcpyDeviceToHost));
        int64_t acc = 0;
        for (int64_t b = 0; b < nblk; ++b) {
            const int32_t v = cnt[b];
            cnt[b] = (int32_t)acc;
            acc += v;
        }
        cnt[nblk] = (int32_t)acc;
        c.nruns = acc;
        PF_CUDA_TRY(cudaMemcpy(c.d_run_off, cnt.data(), sizeof(int32_t) * (nblk + 1),
                               cudaMemcpyHostToDevice));
        PF_CUDA_TRY(cudaMalloc(&c.d_runs, sizeof(int2) * (acc > 0 ? acc : 1)));
        k_p2p_runs<<<(unsigned)nblk, P2P_SETUP_THREADS>>>(L, kb, c.d_q, c.nq, c.nqp, c.d_run_off,
                                                          c.d_runs);
        PF_TRY(pf::launch_status("k_p2p_runs"));
        PF_CUDA_TRY(cudaDeviceSynchronize());
        tally += sizeof(int32_t) * (nblk + 1) + sizeof(int2) * (acc > 0 ? acc : 1);
        // launch order of the blocks: most near-set leaves first, so that the
        // lighter blocks (near the domain edges) fill the end of the launch
        std::vector<int2> runs(acc > 0 ? acc : 1);
        if (acc > 0)
            PF_CUDA_TRY(cudaMemcpy(runs.data(), c.d_runs, sizeof(int2) * acc,
                                   cudaMemcpyDeviceToHost));
        std::vector<int64_t> wgt(nblk, 0);
        for (int64_t b = 0; b < nblk; ++b)
            for (int32_t r = cnt[b]; r < cnt[b + 1]; ++r) wgt[b] += runs[r].y - runs[r].x + 1;
        std::vector<int32_t> order(nblk);
        for (int64_t b = 0; b < nblk; ++b) order[b] = (int32_t)b;
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t a, int32_t b) { return wgt[a] > wgt[b]; });
        PF_TRY(upload(&c.d_blk_order, order, tally));
    }
    c.dev_bytes = tally;
    c.L = L;
    c.kb = kb;
    c.np = np;
    c.ratio = cutoff / w0;
    pf::fmm::separation_key(L, 1.0, c.ratio, THETA, c.sep);
    g_plan_builds.fetch_add(1, std::memory_order_relaxed);
    return PF_OK;
}

struct Sorted {
    uint32_t *key = nullptr;
    int32_t *rank = nullptr, *perm = nullptr, *cnt = nullptr, *start = nullptr;
    double *x = nullptr, *y = nullptr, *g = nullptr;
    float4 *hl = nullptr;
    float *g32 = nullptr;
};

static pf_status sort_points(int64_t n, const double *x, const double *y,
                             const double *g, double x0, double y0, double wl, int L, Sorted &s,
                             int32_t *scan_tmp, uint32_t *skey, int32_t *big, int32_t *big_n,
                             cudaStream_t st) {
    const int64_t nleaf = (int64_t)1 << (2 * L);
    PF_CUDA_TRY(cudaMemsetAsync(s.cnt, 0, sizeof(int32_t) * nleaf, st));
    if (n == 0) {
        PF_CUDA_TRY(cudaMemsetAsync(s.start, 0, sizeof(int32_t) * nleaf, st));
        return PF_OK;
    }
    const unsigned gn = (unsigned)pf::ceil_div(n, 256);
    k_leaf_keys<<<gn, 256, 0, st>>>(x, y, n, x0, y0, wl, L, s.key, s.rank, s.cnt);
    PF_TRY(pf::launch_status("k_leaf_keys"));
    PF_TRY(pf::exclusive_scan_i32(s.cnt, s.start, nleaf, scan_tmp, nullptr, st));
    PF_CUDA_TRY(cudaMemsetAsync(big_n, 0, sizeof(int32_t), st));
    k_place<<<gn, 256, 0, st>>>(n, s.key, s.rank, s.start, s.perm, big, big_n);
    PF_TRY(pf::launch_status("k_place"));
    // leaves above SEG_SMALL particles (dense clusters); the ranks are free now
    PF_TRY(pf::seg_sort_listed(big, big_n, s.start, s.cnt, s.perm, s.rank,
                               n / (pf::SEG_SMALL + 1) + 1, st));
    // the ranks are free again: they receive the final permutation
    k_gather_sorted<<<gn, 256, 0, st>>>(n, s.perm, s.key, s.start, s.cnt, x, y, g, s.rank, s.x,
                                        s.y, s.g, s.hl, s.g32, skey);
    std::swap(s.perm, s.rank);
    return pf::launch_status("k_gather_sorted");
}

static pf_status count_up(int L, int32_t *cnt_all, cudaStream_t st) {
    for (int lc = L; lc > 0;) {
        const int nlev = lc < 4 ? lc : 4;
        const int64_t nblk = (int64_t)1 << (2 * (lc - nlev));
        k_count_up<<<(unsigned)nblk, 256, 0, st>>>(lc, nlev, cnt_all);
        PF_TRY(pf::launch_status("k_count_up"));
        lc -= nlev;
    }
    return PF_OK;
}

struct FmmArgs {
    int64_t ns, nt;
    const double *x, *y, *g, *xt, *yt;
    double ksigmasqr, cutoff, tol;
    int ndirect;
    double *vx, *vy;
};

static size_t fmm_scratch_bytes(const FmmCache &c, int64_t ns, int64_t nt, bool same) {
    const int L = c.L, NP = c.np;
    const int64_t nleaf = (int64_t)1 << (2 * L);
    const int64_t nbox = level_off(L + 1);
    size_t need = 0;
    auto add = [&](size_t b) { need += pf::align256(b); };
    add(4 * ns); add(4 * ns); add(4 * ns);          // key rank perm
    add(8 * ns); add(8 * ns); add(8 * ns);          // x y g
    add(16 * ns); add(4 * ns);                      // hl g32
    if (!same) {
        add(4 * nt); add(4 * nt); add(4 * nt);
        add(8 * nt); add(8 * nt); add(16 * nt);
    }
    add(4 * nt);                                    // sorted target keys
    add(4 * nbox); add(4 * nbox);                   // counts (all levels) src, tgt
    add(4 * nleaf); add(4 * nleaf);                 // starts src, tgt
    add(16 * (size_t)nbox * NP); add(16 * (size_t)nbox * NP);  // M, L
    add(16 * nt);                                   // near velocities
    add(4 * (std::max(ns, nt) / (pf::SEG_SMALL + 1) + 3));  // leaves for the segment sort
    add(4 * (64 + 2 * ((size_t)1 << (2 * (c.L - c.kb)))));  // P2P work distribution
    add(4 * pf::scan_tmp_ints(nleaf));
    return need + 4096;
}

// Run the FMM for one blob set on `st` with a built plan and a scratch region
// of fmm_scratch_bytes(); enqueues kernels only (no host synchronisation).
// ctr: FMM_COUNTERS device counters (P2P pairs, M2L translations, P2P pairs
// evaluated without the exponential), zeroed here.
// ev: 7 events recorded around the phases, or nullptr.
template <int NP>
static pf_status exec_fmm(pf::Bump &sc, const FmmArgs &a, const FmmCache &c, double x0,
                          double y0, double w0, unsigned long long *ctr, cudaEvent_t *ev,
                          cudaStream_t st) {
    const int L = c.L, kb = c.kb;
    const bool same = (a.xt == a.x && a.yt == a.y && a.nt == a.ns);
    const double wl = std::ldexp(w0, -L);
    const int64_t nleaf = (int64_t)1 << (2 * L);
    const int64_t nbox = level_off(L + 1);
    const int64_t ns = a.ns, nt = a.nt;
    auto take = [&](size_t b) { return sc.take(b); };
    Sorted S, T;
    S.key = (uint32_t *)take(4 * ns);
    S.rank = (int32_t *)take(4 * ns);
    S.perm = (int32_t *)take(4 * ns);
    S.x = (double *)take(8 * ns);
    S.y = (double *)take(8 * ns);
    S.g = (double *)take(8 * ns);
    S.hl = (float4 *)take(16 * ns);
    S.g32 = (float *)take(4 * ns);
    if (!same) {
        T.key = (uint32_t *)take(4 * nt);
        T.rank = (int32_t *)take(4 * nt);
        T.perm = (int32_t *)take(4 * nt);
        T.x = (double *)take(8 * nt);
        T.y = (double *)take(8 * nt);
        T.hl = (float4 *)take(16 * nt);
    }
    uint32_t *tkey_sorted = (uint32_t *)take(4 * nt);
    int32_t *scnt_all = (int32_t *)take(4 * nbox);
    int32_t *tcnt_all = (int32_t *)take(4 * nbox);
    S.cnt = scnt_all + level_off(L);
    S.start = (int32_t *)take(4 * nleaf);
    int32_t *tstart = (int32_t *)take(4 * nleaf);
    double2 *M = (double2 *)take(16 * (size_t)nbox * NP);
    double2 *Lc = (double2 *)take(16 * (size_t)nbox * NP);
    double2 *nearv = (double2 *)take(16 * nt);
    // leaves listed for the segment sort: [0] count, [1 ..] leaf ids
    int32_t *big = (int32_t *)take(4 * (std::max(ns, nt) / (pf::SEG_SMALL + 1) + 3));
    // P2P work distribution: counters (64 words), heavy list, group counters
    const int64_t nblk_w = (int64_t)1 << (2 * (L - kb));
    const size_t p2pw_bytes = 4 * (64 + 2 * (size_t)nblk_w);
    unsigned *p2pw_mem = (unsigned *)take(p2pw_bytes);
    int32_t *tmp = (int32_t *)take(4 * pf::scan_tmp_ints(nleaf));
    if (!tmp) {
        pf::set_error("pf_velocity_fmm: scratch layout error");
        return PF_ERR_OOM;
    }
    if (same) {  // targets are the sources: one tree, the target arrays alias the source ones
        T = S;
        tcnt_all = scnt_all;
        tstart = S.start;
    } else {
        T.cnt = tcnt_all + level_off(L);
        T.start = tstart;
    }

    PF_CUDA_TRY(cudaMemsetAsync(ctr, 0, pf::fmmx::FMM_COUNTERS * sizeof(unsigned long long), st));
    auto mark = [&](int k) -> pf_status {
        if (ev) PF_CUDA_TRY(cudaEventRecord(ev[k], st));
        return PF_OK;
    };
    PF_TRY(mark(0));
    // sort sources (and targets)
    // sorted target keys come out of the sorted copies of the targets
    PF_TRY(sort_points(ns, a.x, a.y, a.g, x0, y0, wl, L, S, tmp, same ? tkey_sorted : nullptr,
                       big + 1, big, st));
    if (!same)
        PF_TRY(sort_points(nt, a.xt, a.yt, nullptr, x0, y0, wl, L, T, tmp, tkey_sorted, big + 1,
                           big, st));
    if (same) T = S;  // sort_points replaced S.perm by the final permutation
    PF_TRY(count_up(L, scnt_all, st));
    if (!same) PF_TRY(count_up(L, tcnt_all, st));
    // the near field's description
    const int64_t nblk = (int64_t)1 << (2 * (L - kb));
    P2PDesc pd;
    pd.nblk = nblk;
    pd.kb = kb;
    pd.tstart = tstart;
    pd.tcnt = T.cnt;
    pd.sstart = S.start;
    pd.scnt = S.cnt;
    pd.shl = S.hl;
    pd.sg32 = S.g32;
    pd.thl = T.hl;
    pd.run_off = c.d_run_off;
    pd.runs = c.d_runs;
    pd.order = c.d_blk_order;
    pd.gp = pfd::make_gauss_params(a.ksigmasqr);
    pd.nearv = nearv;
    pd.pairs = ctr;
    pd.work = P2PWork{p2pw_mem, (int32_t *)(p2pw_mem + 64), (int32_t *)(p2pw_mem + 64) + nblk, ns,
                      nt};

    PF_TRY(mark(1));
    // upward pass
    k_p2m<NP><<<(unsigned)pf::ceil_div(4 * nleaf, 128), 128, 0, st>>>(L, x0, y0, wl, S.start, S.cnt,
                                                                 S.x, S.y, S.g, M);
    PF_TRY(pf::launch_status("k_p2m"));
    // parents at levels L-1 .. 2: two levels per launch, one more when odd
    int lp = L - 1;
    for (; lp - 1 >= 2; lp -= 2) {
        const int64_t tasks = ((int64_t)1 << (2 * lp)) / 4;
        k_m2m_tc<NP><<<(unsigned)pf::ceil_div(tasks, TC_THREADS / 32), TC_THREADS, 0, st>>>(
            lp, true, scnt_all, M, c.d_m2m);
        PF_TRY(pf::launch_status("k_m2m_tc"));
    }
    if (lp >= 2) {
        const int64_t tasks = ((int64_t)1 << (2 * lp)) / 4;
        k_m2m_tc<NP><<<(unsigned)pf::ceil_div(tasks, TC_THREADS / 32), TC_THREADS, 0, st>>>(
            lp, false, scnt_all, M, c.d_m2m);
        PF_TRY(pf::launch_status("k_m2m_tc"));
    }
    PF_TRY(mark(2));
    // M2L, all levels >= 2
    const int B = 1 << kb, Bp = B > 2 ? B : 2;
    {
        const int64_t nquad = (nbox - level_off(2)) / 4;  // box quads of levels 2..L
        k_m2l<NP><<<(unsigned)pf::ceil_div(nquad, M2L_THREADS / 32), M2L_THREADS, 0, st>>>(
            L, Bp, nquad, scnt_all, tcnt_all, M, Lc, c.d_far, c.d_far_ptr, c.maxpos, c.d_pw,
            c.d_bin, ctr + 1);
        PF_TRY(pf::launch_status("k_m2l"));
    }
    PF_TRY(mark(3));
    // child levels 3 .. L: two levels per launch, one more when odd
    int lch = 3;
    for (; lch + 1 <= L; lch += 2) {
        const int64_t tasks = ((int64_t)1 << (2 * (lch + 1))) / 16;
        k_l2l_tc<NP><<<(unsigned)pf::ceil_div(tasks, TC_THREADS / 32), TC_THREADS, 0, st>>>(
            lch + 1, true, tcnt_all, Lc, c.d_l2l);
        PF_TRY(pf::launch_status("k_l2l_tc"));
    }
    if (lch <= L) {
        const int64_t tasks = ((int64_t)1 << (2 * lch)) / 16;
        k_l2l_tc<NP><<<(unsigned)pf::ceil_div(tasks, TC_THREADS / 32), TC_THREADS, 0, st>>>(
            lch, false, tcnt_all, Lc, c.d_l2l);
        PF_TRY(pf::launch_status("k_l2l_tc"));
    }
    PF_TRY(mark(4));
    // near field
    {
        PF_CUDA_TRY(cudaMemsetAsync(p2pw_mem, 0, p2pw_bytes, st));
        k_p2p<false><<<(unsigned)nblk, 32, 0, st>>>(pd);
        PF_TRY(pf::launch_status("k_p2p"));
        // the remaining groups of blocks with more than 96 targets (if any)
        const int64_t grid = std::min<int64_t>((int64_t)p2p_sm_count() * P2P_MIN_CTAS, nt / 96 + 1);
        k_p2p<true><<<(unsigned)grid, 32, 0, st>>>(pd);
        PF_TRY(pf::launch_status("k_p2p"));
    }
    PF_TRY(mark(5));
    k_l2p<NP><<<(unsigned)pf::ceil_div(nt, 256), 256, 0, st>>>(nt, L, x0, y0, wl, T.x, T.y,
                                                               tkey_sorted, Lc, nearv, T.perm,
                                                               a.vx, a.vy);
    PF_TRY(pf::launch_status("k_l2p"));
    return mark(6);
}

}  // namespace

// ---------------------------------------------------------------------------
namespace pf {

struct FmmTuning {
    int leaf_level = 0;  // 0 = automatic
    int np = 0;          // 0 = from tol
    int kb = 1;
};
static thread_local FmmTuning g_tune;

int fmmx::np_for_tol(double tol) {
    // Truncation after p+1 terms is bounded by ~theta^(p+1) per translation
    // (theta = 1/2), but the measured end-to-end error is far below that bound:
    // with 16 terms the point-vortex limit (theta-bound at every level) and the
    // Gaussian configurations all stay near 1e-7 at tol = 1e-6, where the FP32
    // near field sets the floor.  So p+1 = log2(1/tol) - 4, rounded up to an
    // instantiated size.
    const int want = (int)std::ceil(std::log2(1.0 / tol)) - 4;
    const int opts[] = {16, 20, 24, 28, 32};
    for (int o : opts)
        if (o >= want) return o;
    return 32;
}

pf_status fmm_exec(const FmmCache &c, double x0, double y0, double w0, Bump &sc,
                   const FmmArgs &a, unsigned long long *ctr, cudaEvent_t *ev, cudaStream_t st) {
    switch (c.np) {
        case 16: return exec_fmm<16>(sc, a, c, x0, y0, w0, ctr, ev, st);
        case 20: return exec_fmm<20>(sc, a, c, x0, y0, w0, ctr, ev, st);
        case 24: return exec_fmm<24>(sc, a, c, x0, y0, w0, ctr, ev, st);
        case 28: return exec_fmm<28>(sc, a, c, x0, y0, w0, ctr, ev, st);
        case 32: return exec_fmm<32>(sc, a, c, x0, y0, w0, ctr, ev, st);
        default:
            // the plan's coefficient arrays are sized for c.np: never run another size on them
            set_error("FMM: %d expansion terms is not an instantiated size (16, 20, 24, 28, 32)",
                      c.np);
            return PF_ERR_INVALID_ARG;
    }
}

// Process-wide cache of read-only plans, shared by every context and thread.
// Tables depend on the geometry only through cutoff / root width, and on that
// ratio only through its separation key (fmm_plan.cuh), so plans are built
// normalised (root width 1) and keyed by (device, L, kb, np, key): a moving
// blob set whose box width drifts keeps its plan until a list changes.
// Least recently used plans are dropped past PF_PLAN_CACHE_BYTES (env,
// default 4 GiB); their device memory is freed when the last user lets go.
struct PlanKey {
    int dev, L, kb, np;
    std::vector<int64_t> sep;
    bool operator<(const PlanKey &o) const {
        if (dev != o.dev) return dev < o.dev;
        if (L != o.L) return L < o.L;
        if (kb != o.kb) return kb < o.kb;
        if (np != o.np) return np < o.np;
        return sep < o.sep;
    }
};
struct PlanCacheStore {
    std::mutex mu;
    std::map<PlanKey, std::pair<std::shared_ptr<FmmCache>, uint64_t>> map;  // plan, last use
    uint64_t tick = 0;
    size_t bytes = 0;
};
static PlanCacheStore &plan_store() {
    static PlanCacheStore *s = new PlanCacheStore();  // never destroyed: outlives the contexts
    return *s;
}
static size_t plan_budget() {
    const char *e = getenv("PF_PLAN_CACHE_BYTES");
    return e ? (size_t)strtoull(e, nullptr, 10) : ((size_t)4 << 30);
}

pf_status shared_plan(int dev, int L, int kb, int np, double ratio,
                      std::shared_ptr<FmmCache> *out) {
    PlanCacheStore &ps = plan_store();
    PlanKey key{dev, L, kb, np, {}};
    pf::fmm::separation_key(L, 1.0, ratio, THETA, key.sep);
    std::lock_guard<std::mutex> lock(ps.mu);
    auto it = ps.map.find(key);
    if (it != ps.map.end()) {
        it->second.second = ++ps.tick;
        *out = it->second.first;
        return PF_OK;
    }
    auto c = std::shared_ptr<FmmCache>(new FmmCache(), [](FmmCache *p) {
        p->release();
        delete p;
    });
    PF_TRY(build_cache(*c, L, kb, np, 1.0, ratio));
    const size_t b = c->bytes();
    while (!ps.map.empty() && ps.bytes + b > plan_budget()) {
        auto old = ps.map.begin();
        for (auto j = ps.map.begin(); j != ps.map.end(); ++j)
            if (j->second.second < old->second.second) old = j;
        ps.bytes -= old->second.first->bytes();
        ps.map.erase(old);
    }
    ps.map[key] = {c, ++ps.tick};
    ps.bytes += b;
    *out = c;
    return PF_OK;
}

}  // namespace pf

extern "C" uint64_t pf_fmm_plan_builds(void) {
    return g_plan_builds.load(std::memory_order_relaxed);
}

extern "C" pf_status pf_fmm_set_tuning(int leaf_level, int expansion_terms, int block_level_drop) {
    pf::clear_error();
    PF_CHECK_ARG(leaf_level == 0 || (leaf_level >= 2 && leaf_level <= MAX_LEVEL),
                 "pf_fmm_set_tuning: leaf level must be 0 (auto) or in [2, %d]", MAX_LEVEL);
    PF_CHECK_ARG(expansion_terms == 0 || expansion_terms == 16 || expansion_terms == 20 ||
                     expansion_terms == 24 || expansion_terms == 28 || expansion_terms == 32,
                 "pf_fmm_set_tuning: expansion terms must be 0 (auto) or one of 16,20,24,28,32");
    PF_CHECK_ARG(block_level_drop >= 0 && block_level_drop <= 2,
                 "pf_fmm_set_tuning: block level drop must be in [0, 2]");
    pf::g_tune.leaf_level = leaf_level;
    pf::g_tune.np = expansion_terms;
    pf::g_tune.kb = block_level_drop;
    return PF_OK;
}

extern "C" pf_status pf_fmm_tree_keys(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                      double x0, double y0, double leaf_width, int leaf_level,
                                      uint32_t *keys, void *stream) {
    PF_RANGE("pf_fmm_tree_keys");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_fmm_tree_keys: NULL context");
    PF_CHECK_ARG(leaf_level >= 1 && leaf_level <= 15, "pf_fmm_tree_keys: leaf level outside [1, 15]");
    PF_CHECK_ARG(leaf_width > 0.0, "pf_fmm_tree_keys: leaf width must be positive");
    PF_CHECK_ARG(n >= 0 && (n == 0 || (x && y && keys)), "pf_fmm_tree_keys: bad arrays");
    pf::DeviceGuard dg(ctx->device);
    if (n == 0) return PF_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_leaf_keys<<<(unsigned)pf::ceil_div(n, 256), 256, 0, st>>>(x, y, n, x0, y0, leaf_width,
                                                               leaf_level, keys, nullptr, nullptr);
    return pf::launch_status("k_leaf_keys");
}

namespace {

// pf_velocity_fmm (box == nullptr: bounding box of sources and targets read
// back from the device, one synchronisation) and pf_velocity_fmm_box (box
// given by the caller, no synchronisation).
pf_status velocity_fmm(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                       const double *g, int64_t n_tgt, const double *xt, const double *yt,
                       double ksigmasqr, double cutoff, double tol, int ndirect, double *vx,
                       double *vy, const double *box, void *stream) {
    PF_CHECK_ARG(ctx != nullptr, "pf_velocity_fmm: NULL context");
    PF_CHECK_ARG(n_src >= 0 && n_tgt >= 0 && n_src < ((int64_t)1 << 31) &&
                     n_tgt < ((int64_t)1 << 31),
                 "pf_velocity_fmm: sizes outside [0, 2^31)");
    PF_CHECK_ARG(ksigmasqr > 0.0 && std::isfinite(ksigmasqr), "pf_velocity_fmm: bad ksigmasqr");
    PF_CHECK_ARG(std::isfinite(cutoff) && cutoff >= 0.0, "pf_velocity_fmm: bad cutoff");
    PF_CHECK_ARG(tol >= 0.0 && tol < 1.0, "pf_velocity_fmm: tol must be in [0, 1)");
    PF_CHECK_ARG(n_src == 0 || (x && y && g), "pf_velocity_fmm: NULL blob array");
    PF_CHECK_ARG(n_tgt == 0 || (xt && yt && vx && vy), "pf_velocity_fmm: NULL target array");
    PF_CHECK_ARG(!box || (std::isfinite(box[0]) && std::isfinite(box[1]) && std::isfinite(box[2]) &&
                          std::isfinite(box[3]) && box[0] <= box[1] && box[2] <= box[3]),
                 "pf_velocity_fmm_box: box must be finite with min <= max");
    pf::DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ctx->last_stream = st;
    pf_fmm_stats &stt = ctx->last_stats;
    memset(&stt, 0, sizeof(stt));
    stt.n_src = n_src;
    stt.n_tgt = n_tgt;
    stt.used_direct = 1;
    if (n_tgt == 0) return PF_OK;
    if (n_src == 0) {
        PF_CUDA_TRY(cudaMemsetAsync(vx, 0, sizeof(double) * n_tgt, st));
        PF_CUDA_TRY(cudaMemsetAsync(vy, 0, sizeof(double) * n_tgt, st));
        return PF_OK;
    }
    if (ndirect < 1) ndirect = 1;
    // leaf level: as the reference's level count, ceil(log4(N / Ndirect))
    int L = pf::g_tune.leaf_level;
    if (L == 0) L = pf::fmmx::auto_level(n_src, ndirect);
    if (tol == 0.0 || L < 3)
        return pf::launch_direct(ctx, n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, vx, vy, st);
    const int np = pf::g_tune.np ? pf::g_tune.np : pf::fmmx::np_for_tol(tol);
    int kb = pf::g_tune.kb;

    // bounding square of sources and targets
    double xmin, xmax, ymin, ymax;
    if (box) {
        xmin = box[0];
        xmax = box[1];
        ymin = box[2];
        ymax = box[3];
    } else {
        PF_TRY(pf::arena_reserve(ctx, 4096));
        BBox *bb = static_cast<BBox *>(pf::arena_take(ctx, sizeof(BBox)));
        k_bbox_init<<<1, 1, 0, st>>>(bb);
        PF_TRY(pf::launch_status("k_bbox_init"));
        const int cap = ctx->num_sms * 8;
        k_bbox<<<(unsigned)std::min<int64_t>(pf::ceil_div(n_src, 256), cap), 256, 0, st>>>(
            x, y, n_src, bb);
        PF_TRY(pf::launch_status("k_bbox"));
        if (!(xt == x && yt == y)) {
            k_bbox<<<(unsigned)std::min<int64_t>(pf::ceil_div(n_tgt, 256), cap), 256, 0, st>>>(
                xt, yt, n_tgt, bb);
            PF_TRY(pf::launch_status("k_bbox"));
        }
        BBox hb;
        PF_CUDA_TRY(
            cudaMemcpyAsync(ctx->host_small, bb, sizeof(BBox), cudaMemcpyDeviceToHost, st));
        PF_CUDA_TRY(cudaStreamSynchronize(st));
        memcpy(&hb, ctx->host_small, sizeof(BBox));
        if (hb.bad) {
            pf::set_error("pf_velocity_fmm: NaN or Inf coordinate");
            return PF_ERR_NAN_INPUT;
        }
        xmin = unord_d(hb.mnx);
        xmax = unord_d(hb.mxx);
        ymin = unord_d(hb.mny);
        ymax = unord_d(hb.mxy);
    }
    double w0 = std::max(xmax - xmin, ymax - ymin);
    if (!(w0 > 0.0)) w0 = 1.0;
    w0 *= 1.0 + 1e-9;
    // the cutoff sets a floor on the leaf width: P2P blocks must stay bounded
    std::shared_ptr<FmmCache> cache;
    for (;;) {
        PF_TRY(pf::shared_plan(ctx->device, L, kb, np, cutoff / w0, &cache));
        if (cache->nqp <= P2P_QMAX) break;
        if (L <= 3) return pf::launch_direct(ctx, n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, vx, vy, st);
        --L;  // cutoff too large for this leaf width: coarser leaves
    }
    ctx->fmm_plan_hold = cache;  // keep the plan alive while this call's kernels run
    FmmArgs a{n_src, n_tgt, x, y, g, xt, yt, ksigmasqr, cutoff, tol, ndirect, vx, vy};
    stt.used_direct = 0;
    stt.leaf_level = L;
    stt.expansion_terms = np;
    stt.block_level_drop = kb;
    const bool same = (xt == x && yt == y && n_tgt == n_src);
    PF_TRY(pf::arena_reserve(ctx, fmm_scratch_bytes(*cache, n_src, n_tgt, same)));
    pf::Bump sc{ctx->arena.base, ctx->arena.cap, 0};
    return pf::fmm_exec(*cache, xmin, ymin, w0, sc, a,
                        reinterpret_cast<unsigned long long *>(ctx->dev_small),
                        ctx->fmm_profile ? ctx->ev : nullptr, st);
}

}  // namespace

extern "C" pf_status pf_velocity_fmm(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                                     const double *g, int64_t n_tgt, const double *xt,
                                     const double *yt, double ksigmasqr, double xopt,
                                     double cutoff, double tol, int ndirect, double *vx,
                                     double *vy, void *stream) {
    PF_RANGE("pf_velocity_fmm");
    pf::clear_error();
    (void)xopt;
    return velocity_fmm(ctx, n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, cutoff, tol, ndirect, vx,
                        vy, nullptr, stream);
}

extern "C" pf_status pf_velocity_fmm_box(pf_ctx *ctx, int64_t n_src, const double *x,
                                         const double *y, const double *g, int64_t n_tgt,
                                         const double *xt, const double *yt, double ksigmasqr,
                                         double xopt, double cutoff, double tol, int ndirect,
                                         const double *box, double *vx, double *vy,
                                         void *stream) {
    PF_RANGE("pf_velocity_fmm_box");
    pf::clear_error();
    (void)xopt;
    PF_CHECK_ARG(box != nullptr, "pf_velocity_fmm_box: NULL box");
    return velocity_fmm(ctx, n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, cutoff, tol, ndirect, vx,
                        vy, box, stream);
}

extern "C" pf_status pf_fmm_profile(pf_ctx *ctx, int enable) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_fmm_profile: NULL context");
    ctx->fmm_profile = enable != 0;
    return PF_OK;
}

extern "C" pf_status pf_fmm_last_stats(pf_ctx *ctx, pf_fmm_stats *out) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr && out != nullptr, "pf_fmm_last_stats: NULL argument");
    pf::DeviceGuard dg(ctx->device);
    pf_fmm_stats s = ctx->last_stats;
    s.ms_sort = s.ms_upward = s.ms_m2l = s.ms_downward = s.ms_p2p = s.ms_l2p = s.ms_total = -1.f;
    if (!s.used_direct) {
        PF_CUDA_TRY(cudaStreamSynchronize(ctx->last_stream));
        unsigned long long c[pf::fmmx::FMM_COUNTERS];
        PF_CUDA_TRY(cudaMemcpy(c, ctx->dev_small, sizeof(c), cudaMemcpyDeviceToHost));
        s.p2p_pairs = (int64_t)c[0];
        s.m2l_translations = (int64_t)c[1];
        s.p2p_pairs_far = (int64_t)c[2];
        if (ctx->fmm_profile) {
            float t[6];
            for (int k = 0; k < 6; ++k) PF_CUDA_TRY(cudaEventElapsedTime(&t[k], ctx->ev[k], ctx->ev[k + 1]));
            s.ms_sort = t[0];
            s.ms_upward = t[1];
            s.ms_m2l = t[2];
            s.ms_downward = t[3];
            s.ms_p2p = t[4];
            s.ms_l2p = t[5];
            PF_CUDA_TRY(cudaEventElapsedTime(&s.ms_total, ctx->ev[0], ctx->ev[6]));
        }
    }
    *out = s;
    return PF_OK;
}

// ---------------------------------------------------------------------------
// internal interface (fmm_api.cuh)
namespace pf {
namespace fmmx {

struct Plan {
    FmmCache c;
    double x0 = 0.0, y0 = 0.0, w0 = 1.0;
};

Plan *plan_new() { return new Plan(); }

void plan_free(Plan *p) {
    if (!p) return;
    p->c.release();
    delete p;
}

pf_status plan_build(Plan *p, int L, int kb, int np, double x0, double y0, double w0,
                     double cutoff, bool *p2p_ok) {
    const double ratio = cutoff / w0;
    std::vector<int64_t> sep;
    pf::fmm::separation_key(L, 1.0, ratio, THETA, sep);
    if (p->c.L != L || p->c.kb != kb || p->c.np != np || p->c.sep != sep)
        PF_TRY(build_cache(p->c, L, kb, np, 1.0, ratio));
    p->x0 = x0;
    p->y0 = y0;
    p->w0 = w0;
    *p2p_ok = p->c.nqp <= P2P_QMAX;
    return PF_OK;
}

int plan_level(const Plan *p) { return p->c.L; }

size_t plan_scratch(const Plan *p, int64_t ns, int64_t nt, bool same) {
    return fmm_scratch_bytes(p->c, ns, nt, same);
}

pf_status plan_exec(const Plan *p, Bump &sc, int64_t ns, const double *x, const double *y,
                    const double *g, int64_t nt, const double *xt, const double *yt,
                    double ksigmasqr, double *vx, double *vy, unsigned long long *ctr,
                    cudaEvent_t *ev, cudaStream_t st) {
    FmmArgs a{ns, nt, x, y, g, xt, yt, ksigmasqr, 0.0, 0.0, 0, vx, vy};
    return fmm_exec(p->c, p->x0, p->y0, p->w0, sc, a, ctr, ev, st);
}

void tuning_get(int *leaf_level, int *np, int *kb) {
    *leaf_level = g_tune.leaf_level;
    *np = g_tune.np;
    *kb = g_tune.kb;
}

void tuning_set(int leaf_level, int np, int kb) {
    g_tune.leaf_level = leaf_level;
    g_tune.np = np;
    g_tune.kb = kb;
}

int auto_level(int64_t ns, int ndirect) {
    if (ndirect < 1) ndirect = 1;
    int L = (int)std::ceil(0.5 * std::log2((double)ns / (double)ndirect));
    return std::min(std::max(L, 0), MAX_LEVEL);
}

}  // namespace fmmx
}  // namespace pf
