/* ref_cutoff_driver.c -- test infrastructure: runs the reference's own
 * cutoff-kernel loops, extracted into _ref/ by the Makefile at build time:
 * the velocity loop of src/cpp/blobs/c/vv2par_C/vv2par_C_cpu.c (constants
 * :99-100, loop :133-151) and the vorticity loop of
 * src/cpp/blobs/c/ww2par_C/ww2par_C_cpu.c (constants :98-99, loop :130-145).
 * The modules' Python-2 C-API wrappers cannot be built here.  Compiled with
 * their flags (-fopenmp -fPIC -O2). */
#include <math.h>

void ref_vv2par_cutoff(int nBlobs, const double *cxB, const double *cyB, const double *cwB,
                       int nTargets, const double *cxT, const double *cyT, double sigmasqr,
                       double *cvx, double *cvy) {
#include "vv2c_consts.inc"
    double xk, yk, s, dx, dy, radius_squared, vxk, vyk;
    int k, m;
    (void)EPS;
#include "vv2c_loop.inc"
#undef PRIVATE_VARS
}

void ref_ww2par_cutoff(int nBlobs, const double *cxB, const double *cyB, const double *cwB,
                       int nTargets, const double *cxT, const double *cyT, double sigmasqr,
                       double *cw) {
#include "ww2c_consts.inc"
    double xk, yk, s, dx, dy, radius, wk;
    int k, m;
    (void)EPS;
#include "ww2c_loop.inc"
#undef PRIVATE_VARS
}
