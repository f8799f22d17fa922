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
// flag is non-null).  No host synchronisation.
pf_status popctl_decide(Bump &sc, int64_t n, const double *g, const int32_t *flag,
                        const PopCtlArgs &pc, cudaStream_t st);

// flag_out[i] = (flag_in ? flag_in[i] != 0 : 1) && !(|g[i]| < state->thr).
// flag_in and flag_out may alias.
pf_status popctl_flags(int64_t n, const double *g, const int32_t *flag_in, const PcState *state,
                       int32_t *flag_out, cudaStream_t st);

// Remesh core (remesh.cu), optionally followed by population control of the
// remeshed cells before they are emitted.  kernel REMESH_M4: M4' weights with
// the Wee coefficient c; REMESH_TUTTY: Tutty weights with c = hNu.
constexpr int REMESH_M4 = 0;
constexpr int REMESH_TUTTY = 1;
size_t remesh_scratch_bytes(int64_t n, int64_t nbx, int64_t nby);
pf_status remesh_core(Bump &sc, int64_t n, const double *x, const double *y, const double *g,
                      double h, double xb0, double yb0, double c, int32_t ixmin, int32_t iymin,
                      int64_t nbx, int64_t nby, int64_t capacity, double *xo, double *yo,
                      double *go, int64_t *ixo, int64_t *iyo, int32_t *total, int32_t *bad,
                      cudaStream_t st, const PopCtlArgs *pc = nullptr, int kernel = REMESH_M4);

}  // namespace pf
