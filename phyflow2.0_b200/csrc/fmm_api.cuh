// fmm_api.cuh -- internal interface of the FMM for other library modules
// (the batch runtime): plans are built on the host once, executions only
// enqueue kernels (no synchronisation, capturable in a CUDA graph).
#pragma once
#include "gauss_pair.cuh"
#include "pf_common.cuh"

namespace pf {
namespace fmmx {

struct Plan;  // tables + device operators for one tree geometry

Plan *plan_new();
void plan_free(Plan *p);
// Build for leaf level L, P2P block drop kb, p+1 = np terms, root box
// [x0, x0+w0] x [y0, y0+w0] and Gaussian cutoff.  Allocates and uploads
// (not capturable).  *p2p_ok = false when the cutoff makes P2P blocks too
// large for this L (use a coarser L).
pf_status plan_build(Plan *p, int L, int kb, int np, double x0, double y0, double w0,
                     double cutoff, bool *p2p_ok);
int plan_level(const Plan *p);
size_t plan_scratch(const Plan *p, int64_t ns, int64_t nt, bool same);
pf_status plan_exec(const Plan *p, Bump &sc, int64_t ns, const double *x, const double *y,
                    const double *g, int64_t nt, const double *xt, const double *yt,
                    double ksigmasqr, double *vx, double *vy, unsigned long long *ctr,
                    cudaEvent_t *ev, cudaStream_t st);
// leaf level from the blob count, as the reference's level count
int auto_level(int64_t ns, int ndirect);
// expansion terms for a tolerance
int np_for_tol(double tol);
// the calling thread's tuning (pf_fmm_set_tuning), to save and restore it
void tuning_get(int *leaf_level, int *np, int *kb);
void tuning_set(int leaf_level, int np, int kb);
constexpr int MAX_LEVEL = 11;
// device counters one FMM call writes (see exec_fmm)
constexpr int FMM_COUNTERS = 3;

// Work-distribution state of the P2P launches of one FMM call, zeroed before
// the first.
struct P2PWork {
    unsigned *heavy_n;   // entries in heavy
    int32_t *heavy;      // blocks with several target groups [nblk]
    int32_t *grp_next;   // groups of each heavy block handed out so far [nblk]
    int64_t ns, nt;      // sorted sources and targets (bounds-checked build)
};

// Everything the near field (P2P) of one FMM call reads and writes: its
// sorted points and leaf tables, the plan's run lists and launch order, the
// kernel parameters and its outputs (the P2P kernels' one argument).
struct P2PDesc {
    int64_t nblk;  // P2P blocks
    int kb;        // block level drop
    const int32_t *tstart, *tcnt, *sstart, *scnt;
    const float4 *shl;
    const float *sg32;
    const float4 *thl;
    const int32_t *run_off;
    const int2 *runs;
    const int32_t *order;
    pfd::GaussParams gp;
    double2 *nearv;
    unsigned long long *pairs;
    P2PWork work;
};

}  // namespace fmmx
}  // namespace pf
