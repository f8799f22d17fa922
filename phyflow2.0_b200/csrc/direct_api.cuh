// direct_api.cuh -- internal interface of the direct sum for the batch runtime.
#pragma once
#include "gauss_pair.cuh"

namespace pf {

struct DirectInstance {
    const double *x, *y, *g;
    int64_t n;
    const double *xt, *yt;
    int64_t nt;
    pfd::GaussParams gp;
    double *vx, *vy;
    int32_t splits;  // source segments (direct_split)
    int64_t seg;     // sources per segment
    float4 *part;    // splits * nt partial sums when splits > 1
};

// Source segmentation of a direct sum: a function of the sizes and of the
// device's resident CTA count only, so the plain and batched paths cut (and
// round) identically.  At most DT_SPLIT_MAX segments of at least
// DT_SPLIT_MIN_SRC sources, whole 32-source chunks (direct.cu).
constexpr int64_t DT_SPLIT_CTAS = 740;  // resident CTAs if the device can't be asked: 5 x 148
constexpr int64_t DT_SPLIT_MIN_SRC = 256;
constexpr int64_t DT_SPLIT_MAX = 64;
struct DirectSplit {
    int splits;
    int64_t seg;
};
DirectSplit direct_split(int64_t ns, int64_t nt);

// targets per work item of the batched kernel
int direct_tile_targets();
// persistent grid size filling every SM
int direct_batch_grid(int num_sms);
// Zeroes *counter_dev and launches the persistent batched direct sum over
// `items` ((instance, tile * splits + segment) pairs in device memory), then
// the reduction of split instances over `reduce_items` ((instance, tile)).
pf_status launch_direct_batch(const DirectInstance *inst_dev, const int2 *items_dev, int n_items,
                              const int2 *reduce_items_dev, int n_reduce, int *counter_dev,
                              int grid, cudaStream_t st);
// cutoff = true: the cutoff kernel g / (r^2 + ksigmasqr), ksigmasqr = sigma^2
pf_status launch_direct(pf_ctx *ctx, int64_t ns, const double *x, const double *y,
                        const double *g, int64_t nt, const double *xt, const double *yt,
                        double ksigmasqr, double *vx, double *vy, cudaStream_t stream,
                        bool cutoff = false);

}  // namespace pf
