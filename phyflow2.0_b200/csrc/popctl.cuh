// popctl.cuh -- population control on the device: the threshold decision of
// PopulationControl (src/python/blobs/base/regrid/_regridding.py:316-330) and
// the keep flags it implies.
#pragma once
#include "pf_common.cuh"

namespace pf {

// Decision state on the device.  `thr` is the threshold finally used (blobs
// with |g| < thr are dropped), `k` the number of decade reductions taken.
struct PcState {
    double thr;
    int32_t decided;
    int32_t k;
    uint32_t done;  // block arrival counter of the current pass (reset by the last block)
    int32_t pad;
};

struct PopCtlArgs {
    double thr_local;   // gThresholdLocal: starting threshold
    double thr_global;  // gThresholdGlobal: admissible dropped circulation
    PcState *state;     // device; receives the decision
};

// Argument checks shared by the entry points (finite, global limit > 0:
// otherwise the reference's loop never ends).
pf_status popctl_check(double thr_local, double thr_global, const char *who);

// Scratch bytes of popctl_decide.
size_t popctl_scratch_bytes();

// Enqueue the decision over the values |g[i]| (only where flag[i] != 0 when
// flag is non-null).  No host synchronisation.  With n_dev non-null the value
// count is *n_dev (a device int64 written by earlier work, at most n); the
// partition of the sums over CTAs then follows *n_dev, so the decision is the
// same as a call with that count given on the host.
pf_status popctl_decide(Bump &sc, int64_t n, const double *g, const int32_t *flag,
                        const PopCtlArgs &pc, cudaStream_t st, const int64_t *n_dev = nullptr);

// flag_out[i] = (flag_in ? flag_in[i] != 0 : 1) && !(|g[i]| < state->thr).
// flag_in and flag_out may alias.
pf_status popctl_flags(int64_t n, const double *g, const int32_t *flag_in, const PcState *state,
                       int32_t *flag_out, cudaStream_t st);

}  // namespace pf
