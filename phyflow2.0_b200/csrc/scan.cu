// scan.cu -- three-pass exclusive scan: per-tile scan + tile totals, one-block
// scan of the totals, add the tile offsets.  Warp-shuffle inclusive scans
// inside each tile; SCAN_ITEMS consecutive elements per thread (coalesced as
// int4).  Deterministic (integer).
#include "scan.cuh"

namespace {

using pf::SCAN_ITEMS;
using pf::SCAN_THREADS;
using pf::SCAN_TILE;

__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ int block_excl_scan(int v, int *s_warp, int *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = warp_incl_scan(v);
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int w = (lane < (blockDim.x >> 5)) ? s_warp[lane] : 0;
        int wi = warp_incl_scan(w);
        s_warp[lane] = wi - w;
        if (lane == 31) s_warp[32] = wi;
    }
    __syncthreads();
    int ex = inc - v + s_warp[wid];
    *total = s_warp[32];
    __syncthreads();
    return ex;
}

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_tiles(const int32_t *__restrict__ in, int32_t *__restrict__ out, int64_t len,
             int32_t *__restrict__ tile_tot) {
    __shared__ int s_warp[33];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < len) ? in[base + k] : 0;
        sum += v[k];
    }
    int tot;
    int ex = block_excl_scan(sum, s_warp, &tot);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < len) out[base + k] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0) tile_tot[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_totals(int32_t *__restrict__ tot, int64_t ntiles, int32_t *__restrict__ total_dev) {
    __shared__ int s_warp[33];
    int carry = 0;
    for (int64_t b0 = 0; b0 < ntiles; b0 += SCAN_THREADS) {
        const int64_t i = b0 + threadIdx.x;
        int v = (i < ntiles) ? tot[i] : 0;
        int t;
        int ex = block_excl_scan(v, s_warp, &t);
        if (i < ntiles) tot[i] = ex + carry;
        carry += t;
    }
    if (threadIdx.x == 0 && total_dev) *total_dev = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_add(int32_t *__restrict__ out, int64_t len, const int32_t *__restrict__ tile_off) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    const int off = tile_off[blockIdx.x];
    if (off == 0) return;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < len) out[base + k] += off;
}

}  // namespace

namespace pf {

pf_status exclusive_scan_i32(const int32_t *in, int32_t *out, int64_t len, int32_t *tmp,
                             int32_t *total_dev, cudaStream_t st) {
    if (len <= 0) {
        if (total_dev) PF_CUDA_TRY(cudaMemsetAsync(total_dev, 0, sizeof(int32_t), st));
        return PF_OK;
    }
    const int64_t ntiles = ceil_div(len, SCAN_TILE);
    if (ntiles > INT32_MAX) {
        set_error("exclusive_scan_i32: length %lld too large", (long long)len);
        return PF_ERR_INVALID_ARG;
    }
    k_scan_tiles<<<(unsigned)ntiles, SCAN_THREADS, 0, st>>>(in, out, len, tmp);
    PF_TRY(launch_status("k_scan_tiles"));
    k_scan_totals<<<1, SCAN_THREADS, 0, st>>>(tmp, ntiles, total_dev);
    PF_TRY(launch_status("k_scan_totals"));
    if (ntiles > 1) {
        k_scan_add<<<(unsigned)ntiles, SCAN_THREADS, 0, st>>>(out, len, tmp);
        PF_TRY(launch_status("k_scan_add"));
    }
    return PF_OK;
}

}  // namespace pf
