// fmm.cu -- 2D FMM for Gaussian blobs (entry point).
#include "pf_common.cuh"

namespace pf {
pf_status launch_direct(int64_t ns, const double *x, const double *y, const double *g,
                        int64_t nt, const double *xt, const double *yt, double ksigmasqr,
                        double *vx, double *vy, cudaStream_t stream);
}

extern "C" pf_status pf_velocity_fmm(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                                     const double *g, int64_t n_tgt, const double *xt,
                                     const double *yt, double ksigmasqr, double xopt,
                                     double cutoff, double tol, int ndirect, double *vx,
                                     double *vy, void *stream) {
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_velocity_fmm: NULL context");
    (void)xopt;
    (void)cutoff;
    (void)ndirect;
    if (tol == 0.0)
        return pf_velocity_direct(ctx, n_src, x, y, g, n_tgt, xt, yt, ksigmasqr, vx, vy, stream);
    pf::set_error("pf_velocity_fmm: FMM path not built yet");
    return PF_ERR_NOT_BUILT;
}
