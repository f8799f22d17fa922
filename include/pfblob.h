/*
 * pfblob.h -- C ABI of the B200 vortex-blob hot path (libpfblob.so).
 *
 * Drop-in boundary for pHyFlow's blob velocity, panel velocity and remesh
 * extension functions.  Plain pointers and sizes only.  Unless stated
 * otherwise every array argument is a DEVICE pointer (cudaMalloc'd or from a
 * caller-owned allocator such as torch), FP64, contiguous, and every call is
 * asynchronous on the CUDA stream passed as `stream` (NULL = legacy default
 * stream).  Calls never abort and never reset the device: failures are
 * reported as a pf_status and a message retrievable with pf_last_error().
 *
 * Ownership: the caller owns inputs and outputs; the library owns scratch in
 * a per-context, grow-only device arena (pf_mem_usage reports its size).  A
 * context may be used from one host thread at a time; use one context per
 * thread for concurrency.
 */
#ifndef PFBLOB_H
#define PFBLOB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pf_status {
    PF_OK = 0,
    PF_ERR_INVALID_ARG = 1, /* bad size, NULL pointer, unsupported option */
    PF_ERR_OOM = 2,         /* device arena could not grow */
    PF_ERR_CUDA = 3,        /* a CUDA runtime call failed (message has the name) */
    PF_ERR_TIMEOUT = 4,     /* a bounded device wait ran out */
    PF_ERR_NAN_INPUT = 5,   /* NaN/Inf in coordinates (checked where stated) */
    PF_ERR_CAPACITY = 6,    /* output capacity too small; *_needed says how much */
    PF_ERR_NOT_BUILT = 7    /* the library was built without the requested path */
} pf_status;

/* Method / hardware / kernel constants, same values as pHyFlow's
 * src/python/blobs/blobOptions.py:53-66. */
#define PF_FMM_METHOD 0
#define PF_DIRECT_METHOD 1
#define PF_CUTOFF_KERNEL 0
#define PF_GAUSS_KERNEL 1

typedef struct pf_ctx pf_ctx;

/* Create a context bound to CUDA device `device`.  Allocates nothing on the
 * device until the first call that needs scratch. */
pf_status pf_create(int device, pf_ctx **out);
pf_status pf_destroy(pf_ctx *ctx);
/* Message of the last failing call on this host thread ("" if none). */
const char *pf_last_error(void);
/* Bytes currently held by the context's scratch arena. */
pf_status pf_mem_usage(const pf_ctx *ctx, size_t *bytes);
/* Release the context's scratch arena (it regrows on demand). */
pf_status pf_trim(pf_ctx *ctx);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int pf_version(void);
/* Process-wide count of kernels this library has launched (all contexts,
 * all threads).  Diagnostic: the difference across a region is the number of
 * library kernels enqueued in it. */
uint64_t pf_kernel_launches(void);

/* ---------------------------------------------------------------------------
 * Gaussian-blob Biot-Savart velocity by direct summation, FP32 arithmetic with
 * hi/lo-split coordinates and compensated accumulation, FP64 in and out.
 *
 *   v_k = 1/(2 pi) sum_m g_m (-dy, dx) / r2 * (1 - exp(-r2/ksigmasqr)),
 *   r2 = dx^2 + dy^2 + 1e-12,  (dx, dy) = target_k - blob_m
 *
 * Replaces vv2parGauss_gpu  (src/cpp/blobs/cuda/vv2parGauss_gpu/
 *   vv2parGauss_py_gpu.cu:104-206, kernel vv2parGauss_device.cu:107-162) and
 *   vv2parGauss_C_cpu (src/cpp/blobs/c/vv2parGauss_C/vv2parGauss_C_cpu.c:89-160),
 * reached from _velocity_direct_{cpu,gpu}_gauss
 *   (src/python/blobs/base/induced/_induced.py:339-518).
 * No padding to a block size is required. n_src or n_tgt may be 0.
 * ------------------------------------------------------------------------- */
pf_status pf_velocity_direct(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                             const double *g, int64_t n_tgt, const double *xt,
                             const double *yt, double ksigmasqr, double *vx, double *vy,
                             void *stream);

/* ---------------------------------------------------------------------------
 * Blob velocity by the 2D fast multipole method (uniform quadtree, FP64
 * multipole/local expansions, FP32-compensated near field with the Gaussian
 * kernel).  Arguments as fmm2d_py: sigma-derived xopt/cutoff are computed by
 * the caller as the reference Python layer does (xopt = sqrt(1.2564312086261697
 * * k sigma^2), cutoff = 5 xopt by default); the velocity is returned directly
 * (vx, vy), i.e. already mapped as (-qi/2pi, -qr/2pi).
 * `ndirect` is the target mean leaf occupancy; `tol` the requested accuracy;
 * tol == 0 computes the direct sum.
 *
 * Replaces fmm2d_py (src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm2d_py.cpp:59-186
 *   GPU, :189-316 CPU) -> fmm2dInteract (fmm.cpp:88-304), reached from
 *   _velocity_fmm_{cpu,gpu}_gauss (src/python/blobs/base/induced/_induced.py:169-336).
 * ------------------------------------------------------------------------- */
pf_status pf_velocity_fmm(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                          const double *g, int64_t n_tgt, const double *xt, const double *yt,
                          double ksigmasqr, double xopt, double cutoff, double tol,
                          int ndirect, double *vx, double *vy, void *stream);

/* Tuning of the FMM for the calling host thread (0 = automatic):
 * leaf_level in [2, 11]; expansion_terms (p+1) in {16, 20, 24, 28, 32};
 * block_level_drop in [0, 2] (P2P blocks of 2^drop x 2^drop leaves).  The
 * reference fixes these at build time (FMM_THETA, Ndirect-based level count,
 * p from tol: src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:538-555); here the
 * autotuner and experiments set them at run time. */
pf_status pf_fmm_set_tuning(int leaf_level, int expansion_terms, int block_level_drop);

/* Leaf Morton keys of points for a tree with origin (x0, y0), leaf width
 * `leaf_width` and leaf level `leaf_level` (<= 15): key = interleave(qx, qy)
 * with qx = clamp(floor((x - x0)/leaf_width), 0, 2^L - 1), x in the even
 * bits.  The same kernel sorts the FMM's particles; exported so the integer
 * keys can be checked bit for bit.  keys: device uint32 array of n entries. */
pf_status pf_fmm_tree_keys(pf_ctx *ctx, int64_t n, const double *x, const double *y, double x0,
                           double y0, double leaf_width, int leaf_level, uint32_t *keys,
                           void *stream);

/* ---------------------------------------------------------------------------
 * Host-only (no device work): the interaction offset tables of the FMM tree
 * for leaf level `leaf_level` (root box width `root_width`, boxes at level l
 * of width root_width/2^l), P2P blocks of 2^block_level_drop leaves a side,
 * separation parameter `theta` and Gaussian `cutoff`.  Two same-level boxes
 * at integer offset (i, j) are well separated when (i^2+j^2) theta^2 >= 2 and
 * (sqrt(i^2+j^2) - sqrt 2) w >= cutoff -- the two connectivity checks of the
 * reference FMM (src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:1735-1835,
 * THETACUTOFFCHECK), which replaces its per-box list build
 * (MPexp_connect_CPU_, fmmsort.cpp:792-910) for a uniform tree.
 * Flattened int32 layout:
 *   L, kb; for l = 0..L: n, n (i, j) pairs (near); for l = 1..L: npos, then per
 *   position n, n (i, j) pairs (M2L); then n, n (i, j) pairs (P2P block list).
 * *needed receives the length; PF_ERR_CAPACITY if `capacity` is smaller.
 * ------------------------------------------------------------------------- */
pf_status pf_fmm_lists(int leaf_level, int block_level_drop, double root_width, double cutoff,
                       double theta, int32_t *buf, int64_t capacity, int64_t *needed);

/* ---------------------------------------------------------------------------
 * Constant-strength straight vortex panels -> induced velocity at points,
 * accumulated into (vx, vy) when `accumulate` != 0 (the blob + panel sum of
 * LagrangianSolver.evaluateVelocity, src/python/lagrangian/
 * __lagrangianSolverClass.py:257-263), else overwritten.
 *
 * Replaces _vortexPanel_Cython_cpu.inducedVelocity (src/cpp/panels/cython/
 *   vortexPanel_Cython/_vortexPanel_Cython_cpu.pyx:243-396), reached from
 *   panelSolver.inducedVelocity (src/python/panels/base/panelSolver.py:148-262),
 *   whose GPU branch is not implemented in the reference (:257-258).
 * Panel arrays have m entries (m <= 65536); evaluation arrays n entries.
 * ------------------------------------------------------------------------- */
pf_status pf_panel_velocity(pf_ctx *ctx, int64_t m, const double *gamma, const double *xs,
                            const double *ys, const double *xe, const double *ye,
                            const double *cosa, const double *sina, int64_t n,
                            const double *xv, const double *yv, double *vx, double *vy,
                            int accumulate, void *stream);

/* ---------------------------------------------------------------------------
 * M4' remesh onto the lattice x_i = i h + h/2 + xb0 (same in y), h = sigma *
 * overlap.  Every cell touched by a blob's 4x4 window is emitted, including
 * cells whose summed weight is exactly zero, in (ix, iy) lexicographic order;
 * duplicates are summed in FP64.  `c` is the Wee diffusion coefficient of the
 * M4' weights (0 = plain remesh).
 *
 * Output capacity: the caller passes arrays of `capacity` entries; *n_out
 * (host pointer) receives the number of new blobs.  If capacity is too small
 * the call returns PF_ERR_CAPACITY with *n_out set to the size needed and
 * writes nothing.  ix_out / iy_out (optional, may be NULL) receive the int64
 * lattice indices.  This call synchronises `stream` twice (to read the
 * lattice extent, then the output count).  The context's scratch arena is
 * shared by all calls on that context: calls issued on different streams with
 * one context must be ordered by the caller.
 *
 * Replaces Regrid (src/python/blobs/base/regrid/_regridding.py:36-222) with
 * m4kernel_1d (src/cpp/blobs/c++/interpolation_kernels_1d/
 * _interpolation_kernels_1d.cpp:21-93), reached from Blobs.redistribute
 * (src/python/blobs/__blobsClass.py:828-897) and diffusion_wee
 * (src/python/blobs/base/evolution/_evolution.py:138-235).
 * ------------------------------------------------------------------------- */
pf_status pf_remesh(pf_ctx *ctx, int64_t n, const double *x, const double *y, const double *g,
                    double h, double xb0, double yb0, double c, int64_t capacity,
                    double *x_out, double *y_out, double *g_out, int64_t *ix_out,
                    int64_t *iy_out, int64_t *n_out, void *stream);

/* ---------------------------------------------------------------------------
 * FP64 moments of a blob set, written to the DEVICE array out4:
 * out4 = {sum g, sum g x, sum g y, sum |g|}, in a fixed reduction order
 * (deterministic).  Used for the circulation / linear impulse conservation
 * checks after remesh.  No reference counterpart (the reference checks
 * nothing); listed for the conservation gate.
 * ------------------------------------------------------------------------- */
pf_status pf_moments(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                     const double *g, double *out4, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PFBLOB_H */
