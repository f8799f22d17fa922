// ref_m4_driver.cpp -- C entry point around the reference's own M4' weight loop.
//
// TEST INFRASTRUCTURE ONLY.  The loop of m4kernel_1d
// (src/cpp/blobs/c++/interpolation_kernels_1d/_interpolation_kernels_1d.cpp:74-89)
// is extracted from the reference file by oracle/Makefile into _ref/m4_loop.inc
// and compiled here unchanged, with the module's own flags (its setup.py:
// distutils defaults + -fopenmp).  The boost.python / pyublas shell around it
// cannot be built here; the loop only needs `x.size()`, `x[k]` and
// `weights[k]`, which the two small views below provide over plain arrays.
#include <cmath>
#include <cstddef>
using namespace std;

namespace {
struct InView {
    const double *p;
    size_t n;
    size_t size() const { return n; }
    double operator[](size_t k) const { return p[k]; }
};
struct OutView {
    double *p;
    double &operator[](size_t k) { return p[k]; }
};
}  // namespace

extern "C" void ref_m4kernel_1d(size_t n, const double *xp, double c, double *out) {
    InView x{xp, n};
    OutView weights{out};
#include "m4_loop.inc"
}
