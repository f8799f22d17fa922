// ref_fmm_driver.cpp -- C entry points around the reference's own CPU FMM.
//
// TEST INFRASTRUCTURE ONLY.  Linked with the reference's FMM sources (compiled
// in place from the pHyFlow tree by oracle/Makefile, output in oracle/_ref/)
// so that the tests and the reference arm of the benchmark can run the
// reference's CPU FMM without boost.python.  Mirrors the defaults that the
// reference binding sets before calling fmm2dInteract:
// src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm2d_py.cpp:293-314 (Oseen smoother,
// sortlimits {2,2,1,1,0,0}, eta {2,2}, pot 1, no panels, no channel).
#include <algorithm>
#include "fmm.h"
#include "direct.h"

extern "C" {

// Returns (qr, qi) exactly as fmm2d_py does; the Python layer of the
// reference maps them to vx = -qi/(2pi), vy = -qr/(2pi)
// (src/python/blobs/base/induced/_induced.py:246-251).
void ref_fmm2d(int n, const double *x, const double *y, const double *g,
               int nt, const double *xt, const double *yt, int ndirect,
               double xopt, double cutoff, double tol, double *qr, double *qi)
{
    bool cont = true;
    double channelheight = -1;
    SMOOTHER smooth = OSEEN;
    float sortlimits[] = {2, 2, 1, 1, 0, 0};
    double eta[] = {2, 2};
    int pot = 1;
    std::fill(qr, qr + nt, 0.0);
    std::fill(qi, qi + nt, 0.0);
    if (tol == 0.0) {
        directInteract(n, x, y, g, NULL, nt, xt, yt, NULL, NULL, qr, qi, NULL, 0,
                       pot, smooth, xopt, cutoff, cont, NULL, false);
    } else {
        fmm2dInteract(n, x, y, g, NULL, nt, xt, yt, NULL, NULL, qr, qi, NULL, 0,
                      pot, tol, ndirect, smooth, xopt, cutoff, cont, NULL, false,
                      sortlimits, eta, channelheight);
    }
}

}  // extern "C"
