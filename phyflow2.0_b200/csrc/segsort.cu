// segsort.cu -- one CTA per listed segment: chunks of SEG_CHUNK values sorted
// in shared memory (bitonic network), then runs merged pairwise, level by
// level, each value written straight to its place: its index in its own run
// plus the number of values of the other run below it (binary search; the
// values are distinct, so there are no ties).  O(c log^2 c) work for a
// segment of c values, no atomics, deterministic.
#include "segsort.cuh"

#include <algorithm>
#include <climits>

namespace {

constexpr int SEG_THREADS = 1024;
constexpr int SEG_CHUNK = 4096;  // values sorted in shared memory at a time

// number of values of the sorted run a[0 .. n) below x
__device__ __forceinline__ int count_below(const int32_t *__restrict__ a, int n, int32_t x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(SEG_THREADS)
k_seg_sort(const int32_t *__restrict__ list, const int32_t *__restrict__ list_n,
           const int32_t *__restrict__ start, const int32_t *__restrict__ cnt,
           int32_t *__restrict__ vals, int32_t *__restrict__ tmp) {
    __shared__ int32_t s_v[SEG_CHUNK];
    const int nlist = *list_n;
    for (int k = blockIdx.x; k < nlist; k += gridDim.x) {
        const int id = list[k];
        const int64_t s0 = start[id];
        const int c = cnt[id];
        // 1. sorted chunks
        for (int ch = 0; ch < c; ch += SEG_CHUNK) {
            const int len = min(SEG_CHUNK, c - ch);
            int p = 1;
            while (p < len) p <<= 1;
            for (int i = threadIdx.x; i < p; i += SEG_THREADS)
                s_v[i] = i < len ? vals[s0 + ch + i] : INT_MAX;
            __syncthreads();
            for (int kk = 2; kk <= p; kk <<= 1) {
                for (int j = kk >> 1; j > 0; j >>= 1) {
                    for (int i = threadIdx.x; i < p; i += SEG_THREADS) {
                        const int ij = i ^ j;
                        if (ij > i) {
                            const int32_t a = s_v[i], b = s_v[ij];
                            const bool up = (i & kk) == 0;
                            if ((a > b) == up) {
                                s_v[i] = b;
                                s_v[ij] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            for (int i = threadIdx.x; i < len; i += SEG_THREADS) vals[s0 + ch + i] = s_v[i];
            __syncthreads();
        }
        // 2. merge runs of width w, 2w, ... (vals and tmp alternate)
        int32_t *src = vals + s0, *dst = tmp + s0;
        for (int w = SEG_CHUNK; w < c; w <<= 1) {
            for (int r0 = 0; r0 < c; r0 += 2 * w) {
                const int na = min(w, c - r0), nb = max(0, min(w, c - r0 - w));
                const int32_t *a = src + r0, *b = src + r0 + w;
                for (int i = threadIdx.x; i < na; i += SEG_THREADS)
                    dst[r0 + i + count_below(b, nb, a[i])] = a[i];
                for (int j = threadIdx.x; j < nb; j += SEG_THREADS)
                    dst[r0 + j + count_below(a, na, b[j])] = b[j];
            }
            __syncthreads();
            int32_t *t = src;
            src = dst;
            dst = t;
        }
        if (src != vals + s0) {
            for (int i = threadIdx.x; i < c; i += SEG_THREADS) vals[s0 + i] = src[i];
        }
        __syncthreads();
    }
}

}  // namespace

namespace pf {

pf_status seg_sort_listed(const int32_t *list, const int32_t *list_n, const int32_t *start,
                          const int32_t *cnt, int32_t *vals, int32_t *tmp, int64_t max_segments,
                          cudaStream_t st) {
    if (max_segments <= 0) return PF_OK;
    // a few CTAs suffice (large segments are rare); each loops over the list
    const unsigned grid = (unsigned)std::min<int64_t>(max_segments, 64);
    k_seg_sort<<<grid, SEG_THREADS, 0, st>>>(list, list_n, start, cnt, vals, tmp);
    return launch_status("k_seg_sort");
}

}  // namespace pf
