// scan.cuh -- device-wide exclusive prefix sum of int32 counts (3 passes).
#pragma once
#include "pf_common.cuh"

namespace pf {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Scratch ints needed by exclusive_scan for `len` elements.
inline size_t scan_tmp_ints(int64_t len) { return (size_t)ceil_div(len, SCAN_TILE) + 1; }

// out[i] = sum_{j<i} in[i]; *total_dev (device int, may be null) = sum of all.
// in and out may alias.  `tmp` holds scan_tmp_ints(len) ints.
pf_status exclusive_scan_i32(const int32_t *in, int32_t *out, int64_t len, int32_t *tmp,
                             int32_t *total_dev, cudaStream_t st);

}  // namespace pf
