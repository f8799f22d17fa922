// step.cu -- one step of a resident blob set in a single call: the induced
// velocity at the blobs (FMM on a known tree box, or the direct sum) and the
// M4' remesh with the window found on the device, with no host
// synchronisation.  A serving loop makes one call per request instead of a
// dozen small ones.
#include <cmath>

#include "fmm_api.cuh"

extern "C" pf_status pf_blob_step(pf_ctx *ctx, const pf_step *s, void *stream) {
    PF_RANGE("pf_blob_step");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_blob_step: NULL context");
    PF_CHECK_ARG(s != nullptr, "pf_blob_step: NULL step");
    PF_CHECK_ARG(s->method == PF_FMM_METHOD || s->method == PF_DIRECT_METHOD,
                 "pf_blob_step: method must be PF_FMM_METHOD or PF_DIRECT_METHOD");
    PF_CHECK_ARG(s->leaf_level == 0 ||
                     (s->leaf_level >= 2 && s->leaf_level <= pf::fmmx::MAX_LEVEL),
                 "pf_blob_step: leaf level must be 0 (auto) or in [2, %d]", pf::fmmx::MAX_LEVEL);
    PF_CHECK_ARG(s->n >= 0 && s->n < ((int64_t)1 << 31), "pf_blob_step: bad n");
    if (s->method == PF_DIRECT_METHOD) {
        PF_TRY(pf_velocity_direct(ctx, s->n, s->x, s->y, s->g, s->n, s->x, s->y, s->ksigmasqr,
                                  s->vx, s->vy, stream));
    } else {
        int L0, np0, kb0;
        pf::fmmx::tuning_get(&L0, &np0, &kb0);
        pf::fmmx::tuning_set(s->leaf_level, 0, 1);
        const pf_status st = pf_velocity_fmm_box(ctx, s->n, s->x, s->y, s->g, s->n, s->x, s->y,
                                                 s->ksigmasqr, s->xopt, s->cutoff, s->tol, 35,
                                                 s->box, s->vx, s->vy, stream);
        pf::fmmx::tuning_set(L0, np0, kb0);
        PF_TRY(st);
    }
    return pf_remesh_async(ctx, s->n, s->x, s->y, s->g, s->h, s->xb0, s->yb0, s->c,
                           s->max_base_cells, s->capacity, s->x_out, s->y_out, s->g_out, nullptr,
                           nullptr, s->n_out_dev, s->status_dev, nullptr, s->moments_dev,
                           stream);
}
