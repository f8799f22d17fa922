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
};

// targets per work item of the batched kernel
int direct_tile_targets();
// persistent grid size filling every SM
int direct_batch_grid(int num_sms);
// Zeroes *counter_dev and launches the persistent batched direct sum over
// `items` ((instance, target tile) pairs in device memory).
pf_status launch_direct_batch(const DirectInstance *inst_dev, const int2 *items_dev, int n_items,
                              int *counter_dev, int grid, cudaStream_t st);
pf_status launch_direct(int64_t ns, const double *x, const double *y, const double *g,
                        int64_t nt, const double *xt, const double *yt, double ksigmasqr,
                        double *vx, double *vy, cudaStream_t stream);

}  // namespace pf
