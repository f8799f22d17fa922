// segsort.cuh -- ascending sort of listed segments of distinct int32 values,
// one CTA per segment, for the large leaves / cells that the per-thread
// insertion sorts of the counting sorts leave alone.
#pragma once
#include "pf_common.cuh"

namespace pf {

// Segments longer than this are sorted by seg_sort_listed; shorter ones by
// the callers' per-thread insertion sorts.
constexpr int SEG_SMALL = 64;

// Sort vals[start[id] .. start[id] + cnt[id]) for every id = list[k],
// k < *list_n (device count).  The values of a segment must be distinct.
// tmp: scratch with the same indexing as vals (only the listed segments'
// ranges are used).  max_segments bounds *list_n (grid size).
pf_status seg_sort_listed(const int32_t *list, const int32_t *list_n, const int32_t *start,
                          const int32_t *cnt, int32_t *vals, int32_t *tmp, int64_t max_segments,
                          cudaStream_t st);

}  // namespace pf
