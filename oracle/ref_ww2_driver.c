/* ref_ww2_driver.c -- test infrastructure: runs the reference's own induced
 * vorticity loop (src/cpp/blobs/c/ww2parGauss_C/ww2parGauss_C_cpu.c:99-101 for
 * its constants, :131-145 for the loop), extracted into _ref/ by the Makefile
 * at build time; the module's Python-2 C-API wrapper cannot be built here.
 * Compiled with that module's flags (-fopenmp -fPIC -O3). */
#include <math.h>

void ref_ww2par_gauss(int nBlobs, const double *cxB, const double *cyB, const double *cwB,
                      int nTargets, const double *cxT, const double *cyT, double ksigmasqr,
                      double *cw) {
#include "ww2_consts.inc"
    double s, dx, dy, radius_squared;
    double wk;
    int k, m;
    (void)s;
#include "ww2_loop.inc"
}
